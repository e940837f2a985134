"""Nuclear-gradient oracle (oracle/grad.py) checked on the CPU.

The reference's gradient (nanoDFT.py:403-477) has no grid-response terms; with the grid frozen
at the reference geometry the converged SCF energy is variational in the density at every
geometry, so its derivative equals the fixed-density derivative minus <dme0, dS/dR> -- the
oracle's formula.  Finite differences of fully re-converged SCF energies on the frozen grid
therefore pin the oracle independently of how it is evaluated."""
import numpy as np

from oracle import eri as oeri
from oracle import grad as ograd
from oracle import rks
from b200dft.mole import Mole, methane
from b200dft.int1e import int1e
from b200dft.grids import build_grid
from b200dft.guess import minao


def _scf(mol, coords, w, D0=None, its=60):
    S, T, V = int1e(mol)
    s8 = oeri.eri_s8(mol)
    ao = rks.ao_values(mol, coords)
    D0 = minao(mol) if D0 is None else D0
    return rks.scf(S, T, V, D0, s8, ao, w, mol.nelectron // 2, mol.energy_nuc(), its=its)


def _grid(mol):
    g = build_grid(mol, 0)
    return np.ascontiguousarray(g.coords), np.ascontiguousarray(g.weights)


def test_gradient_matches_frozen_grid_energy_differences():
    mol = Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7532 -0.4792")
    coords, w = _grid(mol)
    r = _scf(mol, coords, w)
    g = ograd.gradient(mol, r["mo_coeff"], r["mo_energy"], coords, w)
    h = 1e-4
    D = r["logs"][-1, 0]
    fd = np.zeros_like(g)
    for a in range(mol.natm):
        for x in range(3):
            Ep = _scf(ograd._displaced(mol, a, x, h), coords, w, D0=D)["energies"][-1, 0]
            Em = _scf(ograd._displaced(mol, a, x, -h), coords, w, D0=D)["energies"][-1, 0]
            fd[a, x] = (Ep - Em) / (2 * h)
    assert np.abs(g).max() > 1e-2                    # a geometry away from equilibrium
    np.testing.assert_allclose(g, fd, atol=2e-7, rtol=0)          # measured: 3e-8


def test_gradient_methane_symmetry():
    # CH4 along (+-1, +-1, +-1): the level-0 grid (Lebedev rules) keeps the tetrahedral symmetry,
    # so the carbon force vanishes and the four H forces are equal and along their bonds
    mol = Mole(methane(1.12))
    coords, w = _grid(mol)
    r = _scf(mol, coords, w)
    g = ograd.gradient(mol, r["mo_coeff"], r["mo_energy"], coords, w)
    assert np.abs(g[0]).max() < 1e-6
    u = mol.coords[1:] - mol.coords[0]
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    along = (g[1:] * u).sum(1)
    np.testing.assert_allclose(along, along[0], atol=1e-6, rtol=0)
    np.testing.assert_allclose(g[1:] - along[:, None] * u, 0.0, atol=1e-6)
    assert along[0] > 1e-3                           # stretched C-H bonds pull inwards: dE/dr > 0


def test_analytic_gradient_parts_sum_to_the_oracle():
    """one-electron + two-electron + exchange-correlation gradient math (grad_math.cuh, host
    build) plus the nuclear-repulsion derivative (nanoDFT.py:428-438) reproduce the oracle's
    gradient of a converged SCF"""
    import ctypes
    from test_hostcheck import _hc, _p
    hc = _hc()
    mol = Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7532 -0.4792")
    coords, w = _grid(mol)
    r = _scf(mol, coords, w)
    nocc = mol.nelectron // 2
    C = r["mo_coeff"][:, :nocc]
    dm0 = np.ascontiguousarray(2 * C @ C.T)
    dme0 = np.ascontiguousarray(2 * (C * r["mo_energy"][:nocc]) @ C.T)
    atm = np.ascontiguousarray(mol._atm, np.int32)
    bas = np.ascontiguousarray(mol._bas, np.int32)
    env = np.ascontiguousarray(mol._env, np.float64)
    args = (mol.natm, len(bas), _p(atm, ctypes.c_int), _p(bas, ctypes.c_int), _p(env, ctypes.c_double))
    g1, g2, gx = (np.zeros((mol.natm, 3)) for _ in range(3))
    assert hc.b2hc_grad_1e(*args, _p(dm0, ctypes.c_double), _p(dme0, ctypes.c_double), _p(g1, ctypes.c_double)) == 0
    assert hc.b2hc_grad_2e(*args, _p(dm0, ctypes.c_double), ctypes.c_double(rks.HYB), _p(g2, ctypes.c_double)) == 0
    assert hc.b2hc_grad_xc(*args, _p(dm0, ctypes.c_double), ctypes.c_longlong(len(w)), _p(coords, ctypes.c_double),
                           _p(w, ctypes.c_double), _p(gx, ctypes.c_double)) == 0
    Z = mol.charges.astype(np.float64)
    dR = mol.coords[:, None, :] - mol.coords[None, :, :]
    dist = np.linalg.norm(dR, axis=2)
    np.fill_diagonal(dist, np.inf)
    gn = -(Z[:, None, None] * Z[None, :, None] * dR / dist[:, :, None] ** 3).sum(1)
    g = g1 + g2 + gx + gn
    ref = ograd.gradient(mol, r["mo_coeff"], r["mo_energy"], coords, w)
    np.testing.assert_allclose(g, ref, atol=1e-7, rtol=0)
