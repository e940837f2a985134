"""Host AO values on a grid and the AO threshold of the nanoDFT setup.

``eval_ao`` gives the (4, G, nao) array of ``mol.eval_gto('GTOval_sph_deriv1', coords, 4)``
(dft.py:220, nanoDFT.py:220): AO values and their x, y, z derivatives for s / p shells.  The
SCF path generates AO values on the device; the host copy serves the setup option
``ao_threshold`` (nanoDFT.py:221-230), which needs the values before the grid is fixed.
"""
import numpy as np

CHUNK = 8192          # grid points per block (bounds the (G, nao, 3) temporaries)


def eval_ao(mol, coords):
    """(4, G, nao) AO values and x/y/z derivatives at ``coords`` (G x 3, Bohr)."""
    t = mol.ao_table()
    R = mol.coords[t["atom"]]                              # (nao, 3) centres
    is_p = t["l"] == 1
    comp = t["comp"]
    cexp = t["coef"] * t["exps"]
    coords = np.asarray(coords, np.float64).reshape(-1, 3)
    G, N = coords.shape[0], mol.nao
    out = np.empty((4, G, N))
    for g0 in range(0, G, CHUNK):
        d = coords[g0:g0 + CHUNK, None, :] - R[None, :, :]              # (g, nao, 3)
        e = np.exp(-(d * d).sum(-1)[:, :, None] * t["exps"][None])       # (g, nao, nprim)
        rad = (e * t["coef"][None]).sum(-1)                             # sum c exp(-a r^2)
        drad = -2.0 * (e * cexp[None]).sum(-1)                          # its d/d(r^2) x 2
        ang = np.where(is_p[None, :], np.take_along_axis(d, comp[None, :, None], 2)[..., 0], 1.0)
        sl = slice(g0, g0 + d.shape[0])
        out[0, sl] = ang * rad
        for k in range(3):
            out[1 + k, sl] = ang * d[:, :, k] * drad + (is_p & (comp == k))[None, :] * rad
    return out


def threshold_grid(ao, coords, weights, threshold):
    """nanoDFT.py:221-230: AO entries below ``threshold`` in absolute value become 0, and grid
    points where every component of every AO is then 0 are dropped.  Returns the thresholded
    AO array, coordinates and weights of the kept points."""
    ao = np.where(np.abs(ao) < threshold, 0.0, ao)
    keep = np.any(ao != 0.0, axis=(0, 2))
    return np.ascontiguousarray(ao[:, keep]), np.ascontiguousarray(coords[keep]), np.ascontiguousarray(weights[keep])
