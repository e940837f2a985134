"""One-electron matrices (overlap, kinetic, nuclear attraction) for s/p Gaussians.

Replaces the PySCF calls ``mol.intor_symmetric('int1e_ovlp'/'int1e_kin'/'int1e_nuc')``
of dft.py:225-227 and nanoDFT.py:236-238, following the Gaussian-product formulas that
the reference restates in experimental/integrals.py:40-170 (overlap, kinetic via the
Laplacian of the ket, nuclear attraction via Boys functions).  Host-side setup,
vectorised over AO pairs and primitive pairs with numpy.

Every s/p primitive is written as a product of linear factors (d.(r-P) + s) times the
Gaussian product centred at P; Gaussian moments of the (r-P) factors follow from
Isserlis' theorem with variance 1/(2 zeta) per axis.
"""
import itertools
import numpy as np
from scipy.special import gammainc, gamma


def boys(n, t):
    """Boys function F_n(t) = int_0^1 u^{2n} exp(-t u^2) du (vectorised, float64)."""
    t = np.asarray(t, dtype=np.float64)
    out = np.empty_like(t)
    small = t < 1e-7
    ts = t[small]
    out[small] = 1.0 / (2 * n + 1) - ts / (2 * n + 3) + ts * ts / (2 * (2 * n + 5))
    tl = t[~small]
    a = n + 0.5
    out[~small] = gamma(a) * gammainc(a, tl) / (2.0 * tl ** a)
    return out


def _moment(dirs, u):
    """<prod_i d_i.(r-P)> for a Gaussian with per-axis variance u (Isserlis)."""
    if not dirs:
        return 1.0
    if len(dirs) % 2:
        return 0.0
    first, rest = dirs[0], dirs[1:]
    tot = 0.0
    for i, d in enumerate(rest):
        tot = tot + (first * d).sum(-1) * u * _moment(rest[:i] + rest[i + 1:], u)
    return tot


def _factor_product(factors, u):
    """<prod_f (d_f.(r-P) + s_f)> / <1>, expanding over chosen subsets."""
    total = 0.0
    for choice in itertools.product((0, 1), repeat=len(factors)):
        term = 1.0
        dirs = []
        for (d, s), c in zip(factors, choice):
            if c:
                dirs.append(d)
            else:
                term = term * s
        total = total + term * _moment(dirs, u)
    return total


def int1e(mol):
    """Return (S, T, V) as (nao, nao) float64 matrices."""
    tab = mol.ao_table()
    ac = mol.atom_coords()
    A = ac[tab["atom"]]
    isp = (tab["l"] == 1).astype(np.float64)
    dirv = np.zeros((mol.nao, 3))
    dirv[np.where(isp > 0)[0], tab["comp"][isp > 0]] = 1.0
    ex, cf = tab["exps"], tab["coef"]
    a = ex[:, None, :, None]
    b = ex[None, :, None, :]
    cc = cf[:, None, :, None] * cf[None, :, None, :]
    z = a + b
    u = 0.5 / z
    Ai = A[:, None, None, None, :]
    Bj = A[None, :, None, None, :]
    P = (a[..., None] * Ai + b[..., None] * Bj) / z[..., None]
    K = np.exp(-a * b / z * ((Ai - Bj) ** 2).sum(-1))
    PA, PB = P - Ai, P - Bj
    da = dirv[:, None, None, None, :] * np.ones_like(PA)
    db = dirv[None, :, None, None, :] * np.ones_like(PB)
    ia = isp[:, None, None, None]
    jb = isp[None, :, None, None]
    fa = (da, np.where(ia > 0, (PA * da).sum(-1), 1.0))       # factor of AO i (1 for s)
    fb = (db, np.where(jb > 0, (PB * db).sum(-1), 1.0))       # factor of AO j
    s_prim = (np.pi / z) ** 1.5 * K
    ov = _factor_product([fa, fb], u)
    S = (cc * s_prim * ov).sum((2, 3))

    # T = -1/2 <a| lap b>, lap b = (4 b^2 r_B^2 - 2 b (3 + 2 l_b)) b  for l_b <= 1
    r2 = 0.0
    for k in range(3):
        ek = np.zeros(3)
        ek[k] = 1.0
        fk = (ek * np.ones_like(PB), PB[..., k])
        r2 = r2 + _factor_product([fa, fb, fk, fk], u)
    T = (cc * s_prim * (-0.5) * (4 * b * b * r2 - 2 * b * (3 + 2 * jb) * ov)).sum((2, 3))

    # V = sum_C -Z_C (2 pi / z) K sum_h E_h R_h(z, P - C); for linear factors the
    # Hermite expansion is E0 = s_a s_b + d_a.d_b u, E_a = d_a s_b u, E_b = d_b s_a u, E_ab = u^2
    sa, sb = fa[1], fb[1]
    E0 = sa * sb + (da * db).sum(-1) * u
    V = np.zeros((mol.nao, mol.nao))
    for zc, C in zip(mol.atom_charges(), ac):
        X = P - C
        Tz = z * (X * X).sum(-1)
        f0, f1, f2 = (boys(m, Tz) * (-2 * z) ** m for m in range(3))
        Xa = (X * da).sum(-1)
        Xb = (X * db).sum(-1)
        dab = (da * db).sum(-1)
        val = (E0 * f0 + sb * u * Xa * f1 + sa * u * Xb * f1
               + u * u * (dab * f1 + Xa * Xb * f2))
        V += (cc * (-float(zc)) * (2 * np.pi / z) * K * val).sum((2, 3))
    return S, T, V
