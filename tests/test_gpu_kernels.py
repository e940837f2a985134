"""GPU parity: every kernel through the C ABI against the oracle / reference golden data."""
import ctypes
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import eri as oeri, rks
from b200dft.mole import Mole, methane
from b200dft.molgen import config2_molecule, random_molecule
from b200dft.engine import RKSEngine, HostSetup, Plan
from b200dft._lib import lib, check, ptr, stream_handle

pytestmark = pytest.mark.gpu

NAMES = ("h2", "ch4", "water", "tree3")


def _mols():
    gs = [golden(f"eri_ref_{n}.npz") for n in NAMES]
    return [Mole(str(g["atom"]), unit=str(g["unit"])) for g in gs], gs


def _eri(mols, prec, cuda, raw=False):
    """device s8 lists; the plan pads each molecule's list to 32 entries"""
    P = Plan(mols)
    out = torch.full((P.n_eri,), float("nan"), dtype=torch.float64 if prec == 64 else torch.float32,
                     device=cuda)
    check(lib().b2_eri_s8(P.h, prec, ptr(out), stream_handle()), "eri")
    torch.cuda.synchronize()
    v = out.double().cpu().numpy()
    if raw:
        return P, v
    return P, np.concatenate([v[P.eri_off[i]:P.eri_off[i] + oeri.n_s8(int(P.nao[i]))] for i in range(P.nmol)])


def test_eri_s8_fp64_vs_reference(cuda):
    mols, gs = _mols()
    P, v = _eri(mols, 64, cuda)
    assert not np.isnan(v).any()
    ref = np.concatenate([g["s8"] for g in gs])
    err = np.abs(v - ref).max()
    assert err <= 1e-10, err                       # north-star gate: 1e-10 abs


def test_eri_s8_fp32(cuda):
    mols, gs = _mols()
    P, v = _eri(mols, 32, cuda)
    ref = np.concatenate([g["s8"] for g in gs])
    assert np.abs(v - ref).max() < 5e-6


def test_eri_config2_full(cuda):
    g = golden("eri_ref_sample_config2.npz")
    m = Mole(str(g["atom"]))
    P, v = _eri([m], 64, cuda)
    assert len(v) == int(g["n"])
    np.testing.assert_allclose(v[g["idx"]], g["val"], atol=1e-10, rtol=0)
    assert abs(v.sum() - float(g["total"])) <= 1e-9 * abs(float(g["total"]))
    assert abs((v * v).sum() - float(g["sumsq"])) <= 1e-9 * float(g["sumsq"])
    ref = oeri.eri_s8(m)
    assert np.abs(v - ref).max() <= 1e-10


def test_int2e_sph_s8_single(cuda):
    m = Mole(methane())
    out = torch.zeros(oeri.n_s8(m.nao), dtype=torch.float64, device=cuda)
    atm = np.ascontiguousarray(m._atm, np.int32)
    bas = np.ascontiguousarray(m._bas, np.int32)
    env = np.ascontiguousarray(m._env)
    check(lib().b2_int2e_sph_s8(ptr(atm), m.natm, ptr(bas), m.nbas, ptr(env), len(env), 64, ptr(out),
                                stream_handle()), "int2e")
    np.testing.assert_allclose(out.cpu().numpy(), golden("eri_ref_ch4.npz")["s8"], atol=1e-10)


def _sym_random(n, rng):
    a = rng.normal(size=(n, n))
    return (a + a.T) / 2


@pytest.mark.parametrize("prec", [64, 32])
def test_jk_parity(cuda, prec):
    mols, gs = _mols()
    P, v = _eri(mols, prec, cuda, raw=True)
    rng = np.random.default_rng(0)
    Ds = [_sym_random(m.nao, rng) for m in mols]
    eri_t = torch.from_numpy(v).to(cuda).to(torch.float64 if prec == 64 else torch.float32)
    D = torch.from_numpy(P.pack(Ds)).to(cuda)
    J = torch.zeros(P.n_mat, dtype=torch.float64, device=cuda)
    K = torch.zeros_like(J)
    for chunk in (0, 64, 1000):               # several work splits give the same answer
        if chunk:
            P.set_jk_chunk(chunk)
        check(lib().b2_jk_s8(P.h, prec, None, ptr(eri_t), ptr(D), ptr(J), ptr(K), stream_handle()), "jk")
        torch.cuda.synchronize()
        Jh, Kh = J.cpu().numpy(), K.cpu().numpy()
        for mi, (m, g) in enumerate(zip(mols, gs)):
            _, Jr, Kr = rks.jk_from_s8(Ds[mi], g["s8"], m.nao)
            tol = 1e-10 if prec == 64 else 2e-5 * max(1.0, np.abs(Jr).max())
            np.testing.assert_allclose(P.unpack(Jh, mi), Jr, atol=tol)
            np.testing.assert_allclose(P.unpack(Kh, mi), Kr, atol=tol)


@pytest.mark.parametrize("prec", [64, 32])
def test_jk_pairs_parity(cuda, prec):
    # J/K as two products over the s8 list and the exchange list, vs the s8 semantics oracle;
    # inactive molecules keep their previous J/K
    mols, gs = _mols()
    P, v = _eri(mols, prec, cuda, raw=True)
    dt = torch.float64 if prec == 64 else torch.float32
    eri_t = torch.from_numpy(v).to(cuda).to(dt)
    exch = torch.full_like(eri_t, float("nan"))
    check(lib().b2_jk_exchange(P.h, prec, ptr(eri_t), ptr(exch), stream_handle()), "exchange")
    rng = np.random.default_rng(1)
    Ds = [_sym_random(m.nao, rng) for m in mols]
    D = torch.from_numpy(P.pack(Ds)).to(cuda)
    J = torch.full((P.n_mat,), 7.0, dtype=torch.float64, device=cuda)
    K = torch.full_like(J, 7.0)
    active = torch.tensor([1, 0, 1, 1], dtype=torch.int32, device=cuda)
    check(lib().b2_jk_pairs(P.h, prec, ptr(active), ptr(eri_t), ptr(exch), ptr(D), ptr(J), ptr(K),
                            stream_handle()), "jk_pairs")
    torch.cuda.synchronize()
    st = ctypes.c_int(-1)
    check(lib().b2_jk_status(1, ctypes.byref(st)), "b2_jk_status")
    assert st.value == 0                       # no row-group copy wait gave up
    Jh, Kh = J.cpu().numpy(), K.cpu().numpy()
    for mi, (m, g) in enumerate(zip(mols, gs)):
        if mi == 1:
            assert np.all(P.unpack(Jh, mi) == 7.0) and np.all(P.unpack(Kh, mi) == 7.0)
            continue
        _, Jr, Kr = rks.jk_from_s8(Ds[mi], g["s8"], m.nao)
        tol = 1e-10 if prec == 64 else 2e-5 * max(1.0, np.abs(Jr).max())
        np.testing.assert_allclose(P.unpack(Jh, mi), Jr, atol=tol)
        np.testing.assert_allclose(P.unpack(Kh, mi), Kr, atol=tol)
    # exchange list entries: H[(il),(jk)] = (ij|kl) + (ik|jl)
    m, g = mols[2], gs[2]
    N = m.nao
    full = oeri.unpack_s8(g["s8"], N)
    o = int(P.eri_off[2])
    X = exch[o:o + oeri.n_s8(N)].double().cpu().numpy()
    pr = [(i, l) for i in range(N) for l in range(i + 1)]
    e = 0
    for a, (i, l) in enumerate(pr):
        for (j, k) in pr[:a + 1]:
            ref = full[i, j, k, l] + full[i, k, j, l]
            assert abs(X[e] - ref) <= (1e-12 if prec == 64 else 1e-6) * max(1.0, abs(ref))
            e += 1


def test_ao_eval_and_xc(cuda):
    mols = [Mole(methane()), Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7572 -0.4692")]
    eng = RKSEngine(mols, level=0, precision="fp64", setups=[HostSetup(m, 0) for m in mols])
    eng.compute_ao()
    torch.cuda.synchronize()
    ao = eng.ao.cpu().numpy()
    for mi, (m, s) in enumerate(zip(mols, eng.setups)):
        G, N = len(s.weights), m.nao
        a = ao[eng.plan.ao_off[mi]:eng.plan.ao_off[mi] + 4 * G * N].reshape(4, G, N)
        np.testing.assert_allclose(a, rks.ao_values(m, s.coords), atol=1e-12)
    eng.D.copy_(eng.D0)
    for fn in (eng.xc_from_ao, eng.xc):          # stored-AO and on-the-fly-AO paths
        eng.Vxc.zero_()
        fn()
        torch.cuda.synchronize()
        for mi, (m, s) in enumerate(zip(mols, eng.setups)):
            exc, V, _ = rks.exchange_correlation(s.D0, rks.ao_values(m, s.coords), s.weights)
            assert abs(eng.exc[mi].item() - exc) < 1e-10
            np.testing.assert_allclose(eng.plan.unpack(eng.Vxc.cpu().numpy(), mi), V, atol=1e-10)
    eng.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_xc_direct_sizes(cuda, prec):
    # molecules in every orbital bucket (nao 5..65) through the on-the-fly AO path
    rng = np.random.default_rng(4)
    mols = [Mole(random_molecule(rng, k)) for k in (1, 3, 5, 7, 9)]
    setups = [HostSetup(m, 0) for m in mols]
    eng = RKSEngine(mols, level=0, precision=prec, setups=setups)
    eng.D.copy_(eng.D0)
    eng.xc()
    torch.cuda.synchronize()
    tol = 1e-9 if prec == "fp64" else 2e-5
    for mi, (m, s) in enumerate(zip(mols, setups)):
        exc, V, _ = rks.exchange_correlation(s.D0, rks.ao_values(m, s.coords), s.weights)
        assert abs(eng.exc[mi].item() - exc) < tol * max(1, abs(exc))
        np.testing.assert_allclose(eng.plan.unpack(eng.Vxc.cpu().numpy(), mi), V, atol=tol * 10)
    eng.close()


def test_xc_tensor_core_vs_cuda_core(cuda):
    # tcgen05 split-TF32 kernel against the float32 CUDA-core kernel and the float64 oracle,
    # every orbital bucket (nao 5..65), several 128-point tiles per CTA, a converged-like D
    rng = np.random.default_rng(11)
    mols = [Mole(random_molecule(rng, k)) for k in (1, 2, 4, 6, 8, 9)]
    setups = [HostSetup(m, 0) for m in mols]
    eng = RKSEngine(mols, level=0, precision="mixed", setups=setups)
    eng.D.copy_(eng.D0)
    got = {}
    for impl in (1, 2, 0):               # CUDA-core, one-launch tensor-core, per-bucket persistent
        check(lib().b2_plan_set_xc_impl(eng.plan.h, impl), "b2_plan_set_xc_impl")
        eng.xc()
        torch.cuda.synchronize()
        got[impl] = (eng.exc.cpu().numpy().copy(), eng.Vxc.cpu().numpy().copy())
    st = ctypes.c_int(-1)
    check(lib().b2_xc_tc_status(1, ctypes.byref(st)), "b2_xc_tc_status")
    assert st.value == 0
    for mi, (m, s) in enumerate(zip(mols, setups)):
        exc, V, _ = rks.exchange_correlation(s.D0, rks.ao_values(m, s.coords), s.weights)
        Vt = eng.plan.unpack(got[0][1], mi)
        Vs = eng.plan.unpack(got[1][1], mi)
        # float32 quality: relative 2e-6 on E_xc, 2e-5 * max|V| on V
        assert abs(got[0][0][mi] - exc) < 2e-6 * abs(exc)
        np.testing.assert_allclose(Vt, V, atol=2e-5 * np.abs(V).max())
        np.testing.assert_allclose(Vt, Vs, atol=2e-5 * np.abs(V).max())
        np.testing.assert_allclose(Vt, Vt.T, atol=1e-12)
        assert abs(got[2][0][mi] - exc) < 2e-6 * abs(exc)
        np.testing.assert_allclose(eng.plan.unpack(got[2][1], mi), V, atol=2e-5 * np.abs(V).max())
    eng.close()


def test_xc_work_queue_items_active_and_subset(cuda):
    # the per-bucket persistent kernel: several tile counts per work item, inactive molecules
    # left untouched, and a molecule subset (compacted items) give the same V and E_xc
    rng = np.random.default_rng(12)
    mols = [Mole(random_molecule(rng, k)) for k in (9, 1, 5, 3, 7, 2, 8)]
    eng = RKSEngine(mols, level=0, precision="mixed", guess="minao")
    eng.device_setup()
    eng.D.copy_(eng.D0)
    P = eng.plan
    eng.xc()
    torch.cuda.synchronize()
    ref_e, ref_v = eng.exc.cpu().numpy().copy(), eng.Vxc.cpu().numpy().copy()
    for tiles in (1, 3, 16):
        check(lib().b2_plan_set_xc_tiles(P.h, tiles), "b2_plan_set_xc_tiles")
        eng.xc()
        torch.cuda.synchronize()
        np.testing.assert_allclose(eng.exc.cpu().numpy(), ref_e, rtol=1e-6)
        np.testing.assert_allclose(eng.Vxc.cpu().numpy(), ref_v, atol=1e-5 * np.abs(ref_v).max())
    check(lib().b2_plan_set_xc_tiles(P.h, 0), "b2_plan_set_xc_tiles")
    act = torch.tensor([1, 0, 1, 0, 1, 1, 0], dtype=torch.int32, device=cuda)
    eng.Vxc.fill_(7.0)
    eng.exc.fill_(7.0)
    eng.xc(active=act)
    torch.cuda.synchronize()
    V, E = eng.Vxc.cpu().numpy(), eng.exc.cpu().numpy()
    for mi in range(len(mols)):
        if act[mi].item():
            assert abs(E[mi] - ref_e[mi]) <= 1e-6 * abs(ref_e[mi])
            np.testing.assert_allclose(P.unpack(V, mi), P.unpack(ref_v, mi), atol=1e-5 * np.abs(ref_v).max())
        else:
            assert E[mi] == 7.0 and np.all(P.unpack(V, mi) == 7.0)
    idx = np.array([0, 3, 6], np.int32)
    check(lib().b2_plan_set_subset(P.h, ptr(idx), len(idx)), "b2_plan_set_subset")
    sub_act = torch.zeros(len(mols), dtype=torch.int32, device=cuda)
    sub_act[torch.from_numpy(idx.astype(np.int64)).to(cuda)] = 1
    eng.xc(active=sub_act)
    torch.cuda.synchronize()
    check(lib().b2_plan_set_subset(P.h, None, 0), "b2_plan_set_subset")
    for mi in idx:
        np.testing.assert_allclose(P.unpack(eng.Vxc.cpu().numpy(), mi), P.unpack(ref_v, mi),
                                   atol=1e-5 * np.abs(ref_v).max())
    st = ctypes.c_int(-1)
    check(lib().b2_xc_tc_status(1, ctypes.byref(st)), "b2_xc_tc_status")
    assert st.value == 0
    eng.close()


def test_b3lyp_entry(cuda):
    rng = np.random.default_rng(0)
    n = 10000
    rho = np.zeros((4, n))
    rho[0] = 10 ** rng.uniform(-12, 3, n)
    rho[1:] = rng.normal(size=(3, n)) * rho[0] ** (4 / 3)
    r = torch.from_numpy(rho).to(cuda)
    e, vr, vg = (torch.zeros(n, dtype=torch.float64, device=cuda) for _ in range(3))
    check(lib().b2_b3lyp(n, ptr(r), ptr(e), ptr(vr), ptr(vg), stream_handle()), "b3lyp")
    torch.cuda.synchronize()
    e0, vr0, vg0 = rks.b3lyp(rho)
    np.testing.assert_allclose(e.cpu().numpy(), e0, rtol=1e-12)
    np.testing.assert_allclose(vr.cpu().numpy(), vr0, rtol=1e-12)
    np.testing.assert_allclose(vg.cpu().numpy(), vg0, rtol=1e-10)


def test_chol_inv(cuda):
    mols, _ = _mols()
    eng_setups = [HostSetup(m, 0) for m in mols]
    P = Plan(mols)
    S = torch.from_numpy(P.pack([s.S for s in eng_setups])).to(cuda)
    L = torch.zeros_like(S)
    st = torch.zeros(len(mols), dtype=torch.int32, device=cuda)
    check(lib().b2_chol_inv(P.h, ptr(S), ptr(L), ptr(st), stream_handle()), "chol")
    torch.cuda.synchronize()
    assert (st.cpu().numpy() == 0).all()
    for mi, s in enumerate(eng_setups):
        np.testing.assert_allclose(P.unpack(L.cpu().numpy(), mi), s.L_inv, atol=1e-10)
