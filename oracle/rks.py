"""FP64 numpy restatement of the reference's RKS SCF (test infrastructure).

Follows, function by function:
  * AO values + gradients on the grid: ``mol.eval_gto('GTOval_sph_deriv1', coords, 4)``
    (dft.py:220, nanoDFT.py:219-220), evaluated here from the libcint atm/bas/env arrays.
  * B3LYP: b3lyp.py:13-39 with __lda (lda.py:5), __vwn (vwn.py:13-54), __b88 (b88.py:13-29),
    __lyp (lyp.py:13-45).  The reference gets vrho/vgamma with ``jax.value_and_grad``; here
    the same scalar functions are differentiated by the complex-step method, exact to
    machine precision.
  * ``exchange_correlation`` nanoDFT.py:105-123; dense ``get_JK`` nanoDFT.py:129-132;
    ``DIIS`` nanoDFT.py:338-364 (pinv as jnp.linalg.pinv, rcond 10*max(m,n)*eps);
    ``nanoDFT_iteration`` nanoDFT.py:40-102; ``energy`` nanoDFT.py:20-38; ``hlgap`` 366-368.
"""
import numpy as np

from .eri import unpack_s8

HYB = 0.2
EPS = 1e-20
CLIP_MIN, CLIP_MAX = 1e-9, 1e12
FAC = {0: 0.282094791773878143, 1: 0.488602511902919921}


# ------------------------------------------------------------------ AO values on the grid
def ao_values(mol, coords):
    """(4, G, nao): AO values and x/y/z derivatives (GTOval_sph_deriv1 layout)."""
    atm, bas, env = mol._atm, mol._bas, mol._env
    G = coords.shape[0]
    out = []
    for sh in range(bas.shape[0]):
        ia, l, npr, pe, pc = bas[sh, 0], bas[sh, 1], bas[sh, 2], bas[sh, 5], bas[sh, 6]
        R = env[atm[ia, 1]:atm[ia, 1] + 3]
        d = coords - R
        r2 = (d * d).sum(1)
        ex = env[pe:pe + npr]
        cf = env[pc:pc + npr] * FAC[l]
        e = np.exp(-np.outer(r2, ex))                       # (G, npr)
        g0 = e @ cf                                         # sum c exp
        g1 = e @ (cf * ex) * -2.0                           # d/d(r2) * 2 -> coefficient of d
        if l == 0:
            blk = np.zeros((4, G, 1))
            blk[0, :, 0] = g0
            for k in range(3):
                blk[1 + k, :, 0] = g1 * d[:, k]
        else:
            blk = np.zeros((4, G, 3))
            for c in range(3):
                blk[0, :, c] = d[:, c] * g0
                for k in range(3):
                    blk[1 + k, :, c] = (1.0 if k == c else 0.0) * g0 + d[:, c] * d[:, k] * g1
        out.append(blk)
    return np.concatenate(out, axis=2)


# ------------------------------------------------------------------ B3LYP (complex step)
def _lda(x):
    return -np.exp(1 / 3 * np.log(x) - 0.30305460484554375)


def _vwn(n):
    p = np.array([-0.10498, 0.0621813817393097900698817274255, 3.72744, 12.9352])
    f = p[0] * p[2] / (p[0] * p[0] + p[0] * p[2] + p[3]) - 1.0
    f_inv_p1 = 1 / f + 1
    sq = np.sqrt(4.0 * p[3] - p[2] * p[2])
    pre = p[2] * (1.0 / sq - p[0] / ((p[0] * p[0] + p[0] * p[2] + p[3]) * sq / (p[2] + 2.0 * p[0])))
    log_s_c = np.log(3.0 / (4 * np.pi)) / 6
    log_s = -np.log(n) / 6 + log_s_c
    s_2 = np.exp(log_s * 2)
    s = np.exp(log_s)
    z = sq / (2.0 * s + p[2])
    return n * p[1] * (log_s + f * np.log(np.sqrt(s_2 + p[2] * s + p[3]) / (s - p[0]) ** f_inv_p1)
                       + pre * np.arctan(z))


def _b88(a, gaa):
    c1, c2 = 4.0 / 3.0, -8.0 / 3.0
    c3 = (-3.0 / 4.0) * (6.0 / np.pi) ** (1.0 / 3.0) * 2
    d = 0.0042
    log_a = np.log(a / 2)
    na43 = np.exp(log_a * c1)
    chi2 = gaa / 4 * np.exp(log_a * c2)
    chi = np.exp(np.log(chi2) / 2)
    b88 = -(d * na43 * chi2) / (1.0 + 6 * d * chi * np.arcsinh(chi)) * 2
    return c3 * na43 + b88


def _lyp(n, gnn):
    A, B, C, Dd = 0.04918, 0.132, 0.2533, 0.349
    CF = 0.3 * (3.0 * np.pi * np.pi) ** (2.0 / 3.0)
    c0 = 2.0 ** (11.0 / 3.0) * (1 / 2) ** (8 / 3)
    c1 = (1 / 3 + 1 / 8) * 4
    log_n = np.log(n)
    icbrtn = np.exp(log_n * (-1.0 / 3.0))
    P = 1.0 / (1.0 + Dd * icbrtn)
    omega = np.exp(-C * icbrtn) * P
    delta = icbrtn * (C + Dd * P)
    n53 = np.exp(log_n * (-5 / 3))
    return -A * (n * P + B * omega * 1 / 4 * (2 * CF * n * c0 + gnn * (60 - 14.0 * delta) / 36 * n53
                                             - gnn * c1 * n53))


def _cs(f, *args, wrt):
    """complex-step derivative of f w.r.t. argument ``wrt`` (value, derivative)."""
    h = 1e-30
    a = [np.asarray(x, dtype=np.complex128) for x in args]
    scale = np.maximum(np.abs(args[wrt]), 1e-300)
    a[wrt] = a[wrt] + 1j * h * scale
    v = f(*a)
    return v.real, v.imag / (h * scale)


def b3lyp(rho, eps=EPS):
    """b3lyp.py:13-39: rho (4, G) -> (e_xc, vrho, vgamma) per grid point."""
    rho0 = np.clip(rho[0], CLIP_MIN, CLIP_MAX)
    grad = rho[1:4] * 2
    norms = (grad * grad).sum(0) + eps
    e_lda, v_lda = _cs(lambda x: _lda(x) * 0.08, rho0, wrt=0)
    e_vwn, v_vwn = _cs(lambda x: _vwn(x) * 0.19, rho0, wrt=0)
    e_b88, vr_b88 = _cs(lambda x, g: _b88(x, g) * 0.72, rho0, norms, wrt=0)
    _, vn_b88 = _cs(lambda x, g: _b88(x, g) * 0.72, rho0, norms, wrt=1)
    e_lyp, vr_lyp = _cs(lambda x, g: _lyp(x, g) * 0.810, rho0, norms, wrt=0)
    _, vn_lyp = _cs(lambda x, g: _lyp(x, g) * 0.810, rho0, norms, wrt=1)
    e_xc = e_lda + (e_vwn + e_b88 + e_lyp) / rho0
    v_rho = v_lda * 4 * rho0 + v_vwn + vr_b88 + vr_lyp
    v_norm = vn_b88 + vn_lyp
    return e_xc, v_rho, v_norm


# ------------------------------------------------------------------ XC, J/K, DIIS, SCF
def exchange_correlation(D, ao, w):
    """nanoDFT.py:105-123."""
    ao_dm = ao[0] @ D
    rho = (ao_dm[None] * ao).sum(2)
    e_xc, vrho, vgamma = b3lyp(rho, EPS)
    E_xc = float((rho[0] * w * e_xc).sum())
    r = np.concatenate([vrho[None] / 2, 4 * vgamma * rho[1:4]], 0) * w
    V = ao[0].T @ (ao * r[:, :, None]).sum(0)
    return E_xc, V + V.T, rho


def get_JK(D, E):
    """dense branch of nanoDFT.py:129-132 -> diff_JK, J, K."""
    J = np.einsum("ijkl,ji->kl", E, D)
    K = np.einsum("ijkl,jk->il", E, D)
    return J - K / 2 * HYB, J, K


def jk_from_s8(D, s8, nao):
    return get_JK(D, unpack_s8(s8, nao))


def pinv_first_row(B):
    return np.linalg.pinv(B, rcond=10 * max(B.shape) * np.finfo(np.float64).eps)[0, :]


class DIISState:
    def __init__(self, n, space=9):
        self.V = np.zeros((space, n * n))
        self.H = np.zeros((space, n * n))
        self.B = np.zeros((space + 1, space + 1))
        self.B[0, 1:] = self.B[1:, 0] = 1


def diis(i, H, D, S, st):
    """nanoDFT.py:338-364."""
    nd, d = st.V.shape
    head = i % nd
    sdf = S @ D @ H
    err = sdf - sdf.T
    st.V[head] = err.reshape(-1)
    st.H[head] = H.reshape(-1)
    mask = (np.arange(nd) < min(i + 1, nd)).astype(np.float64)
    tmps = (st.V @ err.reshape(-1)) * mask
    st.B[head + 1, 1:] = tmps
    st.B[1:, head + 1] = tmps
    m_ = np.concatenate([[1.0], mask])
    c = pinv_first_row(st.B * m_[:, None] * m_[None, :])
    return (c[1:] @ st.H).reshape(H.shape), float(np.abs(err).max())


def energy(D, H_core, diff_JK, E_xc, E_nuc):
    """nanoDFT.py:20-38 -> [E, E_core, E_J_K/2, E_xc, E_nuc] (Hartree)."""
    E_core = float((D * H_core).sum())
    E_JK = float((D * diff_JK).sum())
    return np.array([E_core + E_JK / 2 + E_xc + E_nuc, E_core, E_JK / 2, E_xc, E_nuc])


def scf(S, T, V, D0, s8, ao, w, nocc, E_nuc, its=20, use_diis=True):
    """nanoDFT's SCF loop (nanoDFT.py:141-160 + 40-102) in FP64.

    Returns dict with per-iteration energies (its, 5) [Ha], D/diff_JK/H logs, DIIS error,
    mo_energy and mo_coeff of the final Hamiltonian.
    """
    N = S.shape[0]
    E = unpack_s8(s8, N)
    L_inv = np.linalg.inv(np.linalg.cholesky(S))
    H_core = T + V
    D = D0.copy()
    E_xc, V_xc, _ = exchange_correlation(D, ao, w)
    diff_JK = get_JK(D, E)[0]
    occ = np.concatenate([np.ones(nocc), np.zeros(N - nocc)])
    st = DIISState(N)
    energies = np.zeros((its, 5))
    logs = np.zeros((its, 3, N, N))
    errs = np.zeros(its)
    for i in range(its):
        H = H_core + diff_JK + V_xc
        if use_diis:
            H, errs[i] = diis(i, H, D, S, st)
        _, vec = np.linalg.eigh(L_inv @ H @ L_inv.T)
        C = L_inv.T @ vec
        D = (C * occ * 2) @ C.T
        E_xc, V_xc, _ = exchange_correlation(D, ao, w)
        diff_JK = get_JK(D, E)[0]
        logs[i] = (D, diff_JK, H)
        energies[i] = energy(D, H_core, diff_JK, E_xc, E_nuc)
    mo_energy, mo_coeff = np.linalg.eigh(L_inv @ logs[-1, 2] @ L_inv.T)
    return dict(energies=energies, logs=logs, diis_err=errs, mo_energy=mo_energy,
                mo_coeff=L_inv.T @ mo_coeff, L_inv=L_inv, H_core=H_core)
