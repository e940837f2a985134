"""Becke-partitioned molecular integration grids.

The reference builds its grids with PySCF (``pyscf.dft.gen_grid.Grids(mol)``,
``grids.level``, dft.py:214-216, nanoDFT.py:215-217) and a partial restatement in
pyscf_utils/build_grid.py:34-135 (Becke partition with the ``original_becke``
3-fold polynomial, box sorting).  PySCF is absent here, so this module is this
project's own equivalent, built from the published constructions:

* radial: Treutler-Ahlrichs M4 mapping of a Chebyshev (second kind) rule
  (Treutler & Ahlrichs, J. Chem. Phys. 102, 346 (1995)), with their per-element xi;
* angular: Lebedev rules of degree 7/11/15 (26/50/86 points; Lebedev & Laikov orbit
  structure, parameters refined here by solving the moment equations) and, above
  degree 15, Gauss-Legendre x trapezoid product rules;
* partition: Becke's fuzzy cells (Becke, J. Chem. Phys. 88, 2547 (1988)) with the
  3-fold polynomial of build_grid.py:34-39 and the atomic-size adjustment of
  Becke's appendix using sqrt of the Bragg-Slater radii (Treutler's variant).

"Grid level" therefore means this module's table ``LEVELS``; the GPU path and
the FP64 oracle always consume the same arrays, so parity is unaffected.
"""
import functools
import math
import numpy as np

from .constants import ANGSTROM_TO_BOHR

# Bragg-Slater radii (Angstrom), H as recommended by Becke (1988)
BRAGG = {1: 0.35, 2: 0.35, 6: 0.70, 7: 0.65, 8: 0.60, 9: 0.50}
# Treutler-Ahlrichs xi
TREUTLER_XI = {1: 0.8, 2: 0.9, 6: 1.1, 7: 0.9, 8: 0.9, 9: 0.9}

# level -> ((n_rad, ang_degree) for H/He, (n_rad, ang_degree) for period 2)
LEVELS = {
    0: ((10, 11), (15, 15)),
    1: ((30, 17), (40, 23)),
    2: ((40, 23), (60, 29)),
    3: ((50, 29), (75, 29)),
    4: ((60, 35), (90, 35)),
}


def _dfact(n):
    return 1.0 if n <= 0 else float(np.prod(np.arange(n, 0, -2, dtype=np.float64)))


def _sphere_moment(a, b, c):
    """(1/4pi) int x^2a y^2b z^2c dOmega."""
    return _dfact(2 * a - 1) * _dfact(2 * b - 1) * _dfact(2 * c - 1) / _dfact(2 * (a + b + c) + 1)


def _orbit(kind, p=None):
    """Points of an octahedral orbit."""
    pts = set()
    if kind == "a1":
        base = [(1.0, 0.0, 0.0)]
    elif kind == "a2":
        s = 1 / math.sqrt(2.0)
        base = [(0.0, s, s)]
    elif kind == "a3":
        s = 1 / math.sqrt(3.0)
        base = [(s, s, s)]
    elif kind == "b":
        l = p
        m = math.sqrt(max(0.0, 1 - 2 * l * l))
        base = [(l, l, m)]
    elif kind == "c":
        q = math.sqrt(max(0.0, 1 - p * p))
        base = [(p, q, 0.0)]
    else:
        raise ValueError(kind)
    import itertools
    for b in base:
        for perm in itertools.permutations(b):
            for sx in (1, -1):
                for sy in (1, -1):
                    for sz in (1, -1):
                        pts.add((round(sx * perm[0], 15) + 0.0, round(sy * perm[1], 15) + 0.0,
                                 round(sz * perm[2], 15) + 0.0))
    return np.array(sorted(pts))


# orbit structure and starting values (weights normalised to sum 1)
_LEBEDEV_SEED = {
    26: [("a1", None, 1 / 21), ("a2", None, 4 / 105), ("a3", None, 9 / 280)],
    50: [("a1", None, 4 / 315), ("a2", None, 64 / 2835), ("a3", None, 27 / 1280),
         ("b", 0.3015113445777636, 14641 / 725760)],
    86: [("a1", None, 0.01154401154401154), ("a3", None, 0.01194390908585628),
         ("b", 0.3696028464541502, 0.01111055571060340),
         ("b", 0.6943540066026664, 0.01187650129453714),
         ("c", 0.3742430390903412, 0.01181230374690448)],
}
_LEBEDEV_DEGREE = {26: 7, 50: 11, 86: 15}


def _assemble(seed, params, weights):
    pts, ws = [], []
    k = 0
    for (kind, p0, _), w in zip(seed, weights):
        p = None
        if p0 is not None:
            p = params[k]
            k += 1
        o = _orbit(kind, p)
        pts.append(o)
        ws.append(np.full(len(o), w))
    return np.vstack(pts), np.concatenate(ws)


@functools.lru_cache(maxsize=None)
def lebedev(npts):
    """Lebedev rule with ``npts`` points: (xyz (n,3), weights summing to 1)."""
    seed = _LEBEDEV_SEED[npts]
    deg = _LEBEDEV_DEGREE[npts]
    mons = [(a, b, c) for a in range(deg // 2 + 1) for b in range(a + 1) for c in range(b + 1)
            if 2 * (a + b + c) <= deg]
    target = np.array([_sphere_moment(*m) for m in mons])
    p0 = [s[1] for s in seed if s[1] is not None]
    w0 = [s[2] for s in seed]

    def resid(x):
        params, weights = x[:len(p0)], x[len(p0):]
        pts, ws = _assemble(seed, params, weights)
        x2, y2, z2 = pts[:, 0] ** 2, pts[:, 1] ** 2, pts[:, 2] ** 2
        return np.array([(ws * x2 ** a * y2 ** b * z2 ** c).sum() for a, b, c in mons]) - target

    x = np.array(p0 + w0, dtype=np.float64)
    for _ in range(30):                       # Gauss-Newton with a numerical Jacobian
        r = resid(x)
        if np.abs(r).max() < 1e-15:
            break
        J = np.empty((len(r), len(x)))
        for i in range(len(x)):
            h = 1e-7 * max(1.0, abs(x[i]))
            xp = x.copy()
            xp[i] += h
            J[:, i] = (resid(xp) - r) / h
        x = x - np.linalg.lstsq(J, r, rcond=None)[0]
    r = resid(x)
    if np.abs(r).max() > 1e-13:
        raise RuntimeError(f"Lebedev {npts}: moment residual {np.abs(r).max():.2e}")
    pts, ws = _assemble(seed, x[:len(p0)], x[len(p0):])
    if len(pts) != npts:
        raise RuntimeError(f"Lebedev {npts}: got {len(pts)} points")
    return pts, ws


@functools.lru_cache(maxsize=None)
def product_rule(degree):
    """Gauss-Legendre (cos theta) x trapezoid (phi) rule exact to ``degree``."""
    nt = degree // 2 + 1
    nphi = degree + 1
    ct, wt = np.polynomial.legendre.leggauss(nt)
    phi = 2 * np.pi * np.arange(nphi) / nphi
    st = np.sqrt(1 - ct * ct)
    x = (st[:, None] * np.cos(phi)[None, :]).ravel()
    y = (st[:, None] * np.sin(phi)[None, :]).ravel()
    z = np.repeat(ct, nphi)
    w = np.repeat(wt / 2.0, nphi) / nphi
    return np.stack([x, y, z], 1), w


def angular_rule(degree):
    for n, d in ((26, 7), (50, 11), (86, 15)):
        if degree <= d:
            return lebedev(n)
    return product_rule(degree)


def treutler_radial(n, xi):
    """Treutler-Ahlrichs M4 radial rule: r_i, w_i (w includes r^2)."""
    i = np.arange(1, n + 1)
    theta = i * np.pi / (n + 1)
    x = np.cos(theta)
    ln2 = math.log(2.0)
    a = 0.6
    r = xi / ln2 * (1 + x) ** a * np.log(2.0 / (1 - x))
    dr = xi / ln2 * (a * (1 + x) ** (a - 1) * np.log(2.0 / (1 - x)) + (1 + x) ** a / (1 - x))
    # Chebyshev 2nd kind: int_{-1}^{1} g(x) dx ~ sum pi/(n+1) sin(theta) g(x)
    w = np.pi / (n + 1) * np.sin(theta) * dr * r * r
    return r[::-1].copy(), w[::-1].copy()


def atomic_grid(z, level):
    """Atom-centred grid (before partitioning): coords (n,3) and weights (4 pi r^2 dr dOmega)."""
    (nr_h, deg_h), (nr_2, deg_2) = LEVELS[level]
    nrad, deg = (nr_h, deg_h) if z <= 2 else (nr_2, deg_2)
    r, wr = treutler_radial(nrad, TREUTLER_XI[z])
    rb = BRAGG[z] * ANGSTROM_TO_BOHR
    coords, weights = [], []
    for ri, wi in zip(r, wr):
        # pruning: the innermost region (r < rb/2) is nearly spherical, use degree 7
        d = 7 if ri < 0.5 * rb else deg
        pts, ws = angular_rule(min(d, deg))
        coords.append(ri * pts)
        weights.append(4 * np.pi * wi * ws)
    return np.vstack(coords), np.concatenate(weights)


def becke_size_adjust(charges):
    """Atomic-size adjustment a_ij of Becke's appendix with sqrt(Bragg) radii."""
    rad = np.sqrt(np.array([BRAGG[int(z)] for z in charges]))
    chi = rad[:, None] / rad[None, :]
    u = (chi - 1) / (chi + 1)
    a = u / (u * u - 1)
    return np.clip(a, -0.5, 0.5)


def becke_partition(coords, atom_coords, charges):
    """Becke cell weights P_A(r) / sum_B P_B(r) for every atom (natm, G)."""
    natm = len(atom_coords)
    dist = np.sqrt(((coords[None, :, :] - atom_coords[:, None, :]) ** 2).sum(-1))
    rab = np.sqrt(((atom_coords[:, None] - atom_coords[None]) ** 2).sum(-1))
    a = becke_size_adjust(charges)
    p = np.ones((natm, coords.shape[0]))
    for i in range(natm):
        for j in range(i):
            mu = (dist[i] - dist[j]) / rab[i, j]
            nu = mu + a[i, j] * (1 - mu * mu)
            g = nu
            for _ in range(3):                         # build_grid.py:34-39
                g = (3 - g * g) * g * 0.5
            p[i] *= 0.5 * (1 - g)
            p[j] *= 0.5 * (1 + g)
    return p / p.sum(0)


class Grids:
    """Drop-in for the fields of ``pyscf.dft.gen_grid.Grids`` the hot path reads."""

    def __init__(self, mol, level=0):
        self.mol = mol
        self.level = level
        self.coords = None
        self.weights = None

    def build(self):
        mol = self.mol
        ac, zs = mol.atom_coords(), mol.atom_charges()
        cs, ws, owner = [], [], []
        for ia in range(mol.natm):
            c, w = atomic_grid(int(zs[ia]), self.level)
            cs.append(c + ac[ia])
            ws.append(w)
            owner.append(np.full(len(w), ia))
        coords = np.vstack(cs)
        w = np.concatenate(ws)
        owner = np.concatenate(owner)
        part = becke_partition(coords, ac, zs)
        self.coords = coords
        self.weights = w * part[owner, np.arange(len(w))]
        self.atom_of_point = owner
        return self

    @property
    def size(self):
        return 0 if self.weights is None else len(self.weights)


def build_grid(mol, level=0):
    return Grids(mol, level).build()
