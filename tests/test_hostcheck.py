"""Kernel arithmetic (the exact __host__ __device__ code of the CUDA kernels, built for the
CPU in libb200dft_hostcheck.so) against the oracle."""
import ctypes
import os
import numpy as np
import pytest

from conftest import golden
from oracle import eri, rks
from b200dft.mole import Mole, methane
from b200dft._lib import HOSTCHECK_PATH


def _hc():
    if not os.path.exists(HOSTCHECK_PATH):
        import subprocess, sys
        subprocess.run([sys.executable, os.path.join(os.path.dirname(os.path.dirname(HOSTCHECK_PATH)),
                        "..", "csrc", "build.py")], check=True)
    return ctypes.CDLL(HOSTCHECK_PATH)


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def hc_eri(mols, prec):
    hc = _hc()
    atm = np.ascontiguousarray(np.concatenate([m._atm for m in mols]), np.int32)
    bas = np.ascontiguousarray(np.concatenate([m._bas for m in mols]), np.int32)
    env = np.concatenate([m._env for m in mols])
    eo = np.cumsum([0] + [len(m._env) for m in mols[:-1]]).astype(np.int64)
    natm = np.array([m.natm for m in mols], np.int32)
    nbas = np.array([m.nbas for m in mols], np.int32)
    out = np.full(sum(eri.n_s8(m.nao) for m in mols), np.nan)
    rc = hc.b2hc_eri_s8(len(mols), _p(natm, ctypes.c_int), _p(nbas, ctypes.c_int), _p(atm, ctypes.c_int),
                        _p(bas, ctypes.c_int), _p(env, ctypes.c_double), _p(eo, ctypes.c_longlong), prec,
                        _p(out, ctypes.c_double))
    assert rc == 0
    return out


def test_eri_math_fp64_vs_reference():
    names = ("h2", "ch4", "water", "tree3")
    gs = [golden(f"eri_ref_{n}.npz") for n in names]
    mols = [Mole(str(g["atom"]), unit=str(g["unit"])) for g in gs]
    v = hc_eri(mols, 64)
    ref = np.concatenate([g["s8"] for g in gs])
    assert not np.isnan(v).any()                     # every s8 slot written exactly by its row
    np.testing.assert_allclose(v, ref, atol=1e-12, rtol=0)


def test_eri_math_fp32():
    g = golden("eri_ref_tree3.npz")
    v = hc_eri([Mole(str(g["atom"]))], 32)
    err = np.abs(v - g["s8"])
    assert err.max() < 5e-6
    assert (err / np.maximum(np.abs(g["s8"]), 1e-2)).max() < 5e-6


def test_boys_device_math():
    hc = _hc()
    F = np.zeros(5)
    for t in np.concatenate([np.linspace(0, 45, 301), [1e-9, 39.99, 40.0, 40.01, 120.0]]):
        hc.b2hc_boys(4, ctypes.c_double(t), _p(F, ctypes.c_double))
        ref = eri.boys(4, t)
        np.testing.assert_allclose(F, ref, rtol=2e-14, atol=1e-17)


def test_b3lyp_device_math():
    hc = _hc()
    rng = np.random.default_rng(0)
    n = 4000
    rho = np.zeros((4, n))
    rho[0] = 10 ** rng.uniform(-12, 3, n)
    rho[1:] = rng.normal(size=(3, n)) * rho[0] ** (4 / 3) * 10 ** rng.uniform(-3, 1, n)
    rho[0, :4] = [0.0, 1e-10, -1e-5, 1e13]           # clipping edge cases (b3lyp.py:15)
    rho = np.ascontiguousarray(rho)
    e, vr, vg = np.zeros(n), np.zeros(n), np.zeros(n)
    hc.b2hc_b3lyp(n, _p(rho, ctypes.c_double), _p(e, ctypes.c_double), _p(vr, ctypes.c_double),
                  _p(vg, ctypes.c_double))
    e0, vr0, vg0 = rks.b3lyp(rho)
    np.testing.assert_allclose(e, e0, rtol=1e-12)
    np.testing.assert_allclose(vr, vr0, rtol=1e-12)
    np.testing.assert_allclose(vg, vg0, rtol=1e-10)


def test_plan_class_starts_without_pair_tables():
    """the device plan counts each molecule's shell pairs per angular class from the shells' l
    alone (its pair tables are built on the GPU); the counts must equal the host pair tables'"""
    from b200dft.molgen import config3_batch
    hc = _hc()
    mols = [Mole(s) for s in config3_batch(48, seed=5)] + [Mole(methane()), Mole("H 0 0 0; H 0 0 0.74")]
    atm = np.ascontiguousarray(np.concatenate([m._atm for m in mols]), np.int32)
    bas = np.ascontiguousarray(np.concatenate([m._bas for m in mols]), np.int32)
    env = np.concatenate([m._env for m in mols])
    eo = np.cumsum([0] + [len(m._env) for m in mols[:-1]]).astype(np.int64)
    natm = np.array([m.natm for m in mols], np.int32)
    nbas = np.array([m.nbas for m in mols], np.int32)
    fast = np.zeros(5 * len(mols), np.int32)
    ref = np.full(5 * len(mols), -1, np.int32)
    rc = hc.b2hc_plan_classes(len(mols), _p(natm, ctypes.c_int), _p(nbas, ctypes.c_int), _p(atm, ctypes.c_int),
                              _p(bas, ctypes.c_int), _p(env, ctypes.c_double), _p(eo, ctypes.c_longlong),
                              _p(fast, ctypes.c_int), _p(ref, ctypes.c_int))
    assert rc == 0
    np.testing.assert_array_equal(fast, ref)
    nsp = nbas.astype(np.int64) * (nbas + 1) // 2
    np.testing.assert_array_equal(fast.reshape(-1, 5)[:, 4], nsp)


def test_two_electron_gradient_vs_finite_differences():
    """the two-electron gradient math (grad_math.cuh, host build) against central differences
    of E_2e = sum (ij|kl) Gamma_ijkl at fixed density, Gamma = 1/2 D_ij D_kl - hyb/4 D_il D_jk,
    with the ERI oracle at the displaced geometries"""
    from oracle import grad as ograd
    hc = _hc()
    for mol in (Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7532 -0.4792"), Mole(methane(1.05))):
        N, hyb = mol.nao, 0.2
        rng = np.random.default_rng(4)
        D = rng.normal(size=(N, N)) * 0.3
        D = np.ascontiguousarray(D + D.T)
        gam = 0.5 * np.einsum("ij,kl->ijkl", D, D) - hyb / 4 * np.einsum("il,jk->ijkl", D, D)
        g = np.zeros((mol.natm, 3))
        atm = np.ascontiguousarray(mol._atm, np.int32)
        bas = np.ascontiguousarray(mol._bas, np.int32)
        env = np.ascontiguousarray(mol._env, np.float64)
        rc = hc.b2hc_grad_2e(mol.natm, len(bas), _p(atm, ctypes.c_int), _p(bas, ctypes.c_int),
                             _p(env, ctypes.c_double), _p(D, ctypes.c_double), ctypes.c_double(hyb),
                             _p(g, ctypes.c_double))
        assert rc == 0
        h = 1e-4
        fd = np.zeros_like(g)
        for a in range(mol.natm):
            for x in range(3):
                e = [float((eri.unpack_s8(eri.eri_s8(ograd._displaced(mol, a, x, s * h)), N) * gam).sum())
                     for s in (1, -1)]
                fd[a, x] = (e[0] - e[1]) / (2 * h)
        assert np.abs(fd).max() > 1e-2
        np.testing.assert_allclose(g, fd, atol=1e-7 * max(1.0, np.abs(fd).max()), rtol=0)
        np.testing.assert_allclose(g.sum(0), 0.0, atol=1e-9)    # translation invariance (exact)


def test_two_electron_gradient_kernel_traversal():
    """the GPU kernels' traversal of the two-electron gradient (canonical shell quartets of the
    float32 ERI work list, degeneracy weights, symmetrised Gamma, class fixed by the task group)
    equals the sum over all ordered quartets, molecule by molecule in a batch"""
    hc = _hc()
    mols = [Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7532 -0.4792"), Mole(methane(1.05)),
            Mole("N 0 0 0; C 0 0 2.6; O 2.1 0 3.9; H 0 1.9 -0.8", unit="Bohr")]
    rng = np.random.default_rng(7)
    Ds, hyb = [], 0.2
    for m in mols:
        X = rng.normal(size=(m.nao, m.nao)) * 0.3
        Ds.append(np.ascontiguousarray(X + X.T))
    atm = np.ascontiguousarray(np.concatenate([m._atm for m in mols]), np.int32)
    bas = np.ascontiguousarray(np.concatenate([m._bas for m in mols]), np.int32)
    env = np.concatenate([m._env for m in mols])
    eo = np.cumsum([0] + [len(m._env) for m in mols[:-1]]).astype(np.int64)
    natm = np.array([m.natm for m in mols], np.int32)
    nbas = np.array([m.nbas for m in mols], np.int32)
    Dp = np.ascontiguousarray(np.concatenate([D.reshape(-1) for D in Ds]))
    g = np.full((int(natm.sum()), 3), np.nan)
    bad = ctypes.c_int(-1)
    rc = hc.b2hc_grad_2e_tasks(len(mols), _p(natm, ctypes.c_int), _p(nbas, ctypes.c_int), _p(atm, ctypes.c_int),
                               _p(bas, ctypes.c_int), _p(env, ctypes.c_double), _p(eo, ctypes.c_longlong),
                               _p(Dp, ctypes.c_double), ctypes.c_double(hyb), _p(g, ctypes.c_double),
                               ctypes.byref(bad))
    assert rc == 0 and bad.value == 0
    a0 = 0
    for m, D in zip(mols, Ds):
        ref = np.zeros((m.natm, 3))
        ma = np.ascontiguousarray(m._atm, np.int32)
        mb = np.ascontiguousarray(m._bas, np.int32)
        me = np.ascontiguousarray(m._env, np.float64)
        assert hc.b2hc_grad_2e(m.natm, len(mb), _p(ma, ctypes.c_int), _p(mb, ctypes.c_int), _p(me, ctypes.c_double),
                               _p(D, ctypes.c_double), ctypes.c_double(hyb), _p(ref, ctypes.c_double)) == 0
        np.testing.assert_allclose(g[a0:a0 + m.natm], ref, atol=1e-10 * max(1.0, np.abs(ref).max()), rtol=0)
        a0 += m.natm


def test_two_electron_gradient_recursion_tables():
    """the step tables the GPU two-electron gradient kernels split over a warp's lanes (target,
    sources, direction, factors, last m of every Obara-Saika step), run in table order on the
    host, give the serial recursion's weighted [e0|f0] sums for every class combination, with the
    bra raised by one and with the ket raised by one"""
    hc = _hc()
    rel = np.full(32, np.nan)
    assert hc.b2hc_grad_vrr_tables(_p(rel, ctypes.c_double)) == 0
    assert np.all(rel < 1e-12), rel


def test_one_electron_gradient_vs_finite_differences():
    """the one-electron gradient math (host build) against central differences of
    <D, T + V_nuc> - <W, S> at fixed D and W, with the host 1e integrals at displaced geometries"""
    from oracle import grad as ograd
    from b200dft.int1e import int1e
    hc = _hc()
    for mol in (Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7532 -0.4792"), Mole(methane(1.05))):
        N = mol.nao
        rng = np.random.default_rng(6)
        D = rng.normal(size=(N, N)) * 0.3
        D = np.ascontiguousarray(D + D.T)
        W = rng.normal(size=(N, N)) * 0.3
        W = np.ascontiguousarray(W + W.T)
        g = np.zeros((mol.natm, 3))
        atm = np.ascontiguousarray(mol._atm, np.int32)
        bas = np.ascontiguousarray(mol._bas, np.int32)
        env = np.ascontiguousarray(mol._env, np.float64)
        rc = hc.b2hc_grad_1e(mol.natm, len(bas), _p(atm, ctypes.c_int), _p(bas, ctypes.c_int),
                             _p(env, ctypes.c_double), _p(D, ctypes.c_double), _p(W, ctypes.c_double),
                             _p(g, ctypes.c_double))
        assert rc == 0
        h = 1e-4
        fd = np.zeros_like(g)
        for a in range(mol.natm):
            for x in range(3):
                e = []
                for s in (1, -1):
                    S, T, V = int1e(ograd._displaced(mol, a, x, s * h))
                    e.append(float((D * (T + V)).sum() - (W * S).sum()))
                fd[a, x] = (e[0] - e[1]) / (2 * h)
        assert np.abs(fd).max() > 1e-2
        np.testing.assert_allclose(g, fd, atol=1e-7 * max(1.0, np.abs(fd).max()), rtol=0)


def test_xc_gradient_vs_finite_differences():
    """the exchange-correlation gradient math (host build) against central differences of the
    oracle's E_xc at fixed density on a fixed grid (the grid does not move with the atoms, as in
    the reference's gradient)"""
    from oracle import grad as ograd
    from b200dft.grids import build_grid
    from b200dft.guess import minao
    hc = _hc()
    mol = Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7532 -0.4792")
    grid = build_grid(mol, 0)
    coords = np.ascontiguousarray(grid.coords, np.float64)
    w = np.ascontiguousarray(grid.weights, np.float64)
    D = np.ascontiguousarray(minao(mol), np.float64)
    g = np.zeros((mol.natm, 3))
    atm = np.ascontiguousarray(mol._atm, np.int32)
    bas = np.ascontiguousarray(mol._bas, np.int32)
    env = np.ascontiguousarray(mol._env, np.float64)
    rc = hc.b2hc_grad_xc(mol.natm, len(bas), _p(atm, ctypes.c_int), _p(bas, ctypes.c_int),
                         _p(env, ctypes.c_double), _p(D, ctypes.c_double), ctypes.c_longlong(len(w)),
                         _p(coords, ctypes.c_double), _p(w, ctypes.c_double), _p(g, ctypes.c_double))
    assert rc == 0
    h = 1e-4
    fd = np.zeros_like(g)
    for a in range(mol.natm):
        for x in range(3):
            e = [rks.exchange_correlation(D, rks.ao_values(ograd._displaced(mol, a, x, s * h), coords), w)[0]
                 for s in (1, -1)]
            fd[a, x] = (e[0] - e[1]) / (2 * h)
    assert np.abs(fd).max() > 1e-2
    np.testing.assert_allclose(g, fd, atol=1e-6 * max(1.0, np.abs(fd).max()), rtol=0)


def test_gradient_math_compiles_for_sm100a(tmp_path):
    """the gradient math is host and device code: it must also build as sm_100a device code (one
    class of the two-electron part here; the library build compiles all sixteen in grad.cu)"""
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    csrc = os.path.join(os.path.dirname(os.path.dirname(HOSTCHECK_PATH)), "..", "csrc")
    src = tmp_path / "k.cu"
    src.write_text(
        '#include "grad_math.cuh"\n'
        "__global__ void k(const B2Shell *s, const double *t, const double *gam, const double *D,\n"
        "                  const double *W, const double *Z, const double *RC, const double *r, double *o) {\n"
        "  double g4[4][3], g2[2][3], f[3], df[3][3], hf[3][6];\n"
        "  b2g_quartet_grad_t<double, 1, 0, 0, 1>(s[0], s[1], s[2], s[3], t, gam, g4);\n"
        "  b2g_pair_grad_1e<double>(s[0], s[1], D, W, 9, 5, Z, RC, t, g2,\n"
        "                           [&](int c, int x, double v) { atomicAdd(o + 3 * c + x, v); });\n"
        "  b2g_ao2<double>(s[0], r, f, df, hf);\n"
        "  o[0] += g4[0][0] + g2[0][0] + f[0] + df[0][0] + hf[0][0];\n"
        "}\n")
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
                        "--expt-relaxed-constexpr", "-I", csrc, "-c", str(src), "-o", str(tmp_path / "k.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
