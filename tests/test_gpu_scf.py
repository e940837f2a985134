"""GPU parity of the SCF loop and the drop-in entry points against the FP64 oracle."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import eri as oeri, rks
from b200dft.mole import Mole, methane
from b200dft.molgen import random_molecule
from b200dft.engine import RKSEngine, HostSetup
from b200dft.int1e import int1e
from b200dft.guess import minao
from b200dft import nanodft, dft
from b200dft.constants import HARTREE_TO_EV

pytestmark = pytest.mark.gpu


def oracle_scf(m, setup, its=20):
    ao = rks.ao_values(m, setup.coords)
    return rks.scf(setup.S, setup.T, setup.V, setup.D0, oeri.eri_s8(m), ao, setup.weights,
                   m.nelectron // 2, setup.E_nuc, its=its)


@pytest.mark.parametrize("name", ["ch4", "water"])
def test_scf_fp64_vs_oracle(cuda, name):
    g = golden(f"scf_oracle_{name}.npz")
    m = Mole(str(g["atom"]), unit=str(g["unit"]))
    eng = RKSEngine([m], level=0, precision="fp64")
    res = eng.run(its=20)
    eng.close()
    E = res["energies"][:, 0, 0]
    assert np.abs(E - g["energies"][:, 0]).max() <= 1e-6           # north-star gate (Ha)
    np.testing.assert_allclose(res["mo_energy"][-1, 0, :m.nao], g["mo_energy"], atol=1e-6)


def test_scf_batch_uneven_fp64(cuda):
    rng = np.random.default_rng(5)
    mols = [Mole(methane()), Mole(random_molecule(rng, 2)), Mole(random_molecule(rng, 3))]
    eng = RKSEngine(mols, level=0, precision="fp64")
    res = eng.run(its=15)
    for mi, m in enumerate(mols):
        ref = oracle_scf(m, HostSetup(m, 0), its=15)
        assert np.abs(res["energies"][:, mi, 0] - ref["energies"][:, 0]).max() <= 1e-6
    eng.close()


def test_scf_mixed_precision(cuda):
    rng = np.random.default_rng(11)
    m = Mole(random_molecule(rng, 4))
    eng = RKSEngine([m], level=0, precision="mixed")
    res = eng.run(its=20)
    eng.close()
    ref = oracle_scf(m, HostSetup(m, 0), its=20)
    assert abs(res["energies"][-1, 0, 0] - ref["energies"][-1, 0]) <= 1e-4   # north-star: 1e-4 Ha


def test_nanodft_dropin(cuda):
    opts, mol_str = nanodft.nanoDFT_options(its=12, mol_str="methane", level=0)
    mol = nanodft.build_mol(mol_str, opts.basis)
    E, (logged, hl, mo_e, mo_c, coords, w) = nanodft.nanoDFT(mol, opts)
    assert E.shape == (12, 5) and logged.shape == (12, 5)
    g = golden("scf_oracle_ch4.npz")
    np.testing.assert_allclose(E[:, 0] / HARTREE_TO_EV, g["energies"][:12, 0], atol=1e-6)
    np.testing.assert_allclose(E, logged, atol=1e-6)                 # host FP64 recompute == device
    # orbitals: C^T S C = 1 and S C = F C e structure
    S, T, V = int1e(mol)
    np.testing.assert_allclose(mo_c.T @ S @ mo_c, np.eye(mol.nao), atol=1e-8)
    assert hl[-1] > 0 and len(w) == len(coords)


def test_dft_dropin(cuda):
    args = dft.get_args(["-its", "10", "-level", "0"])
    m = Mole(methane())
    s = "; ".join(f"{sym} {x} {y} {z}" for sym, (x, y, z) in zip(m.symbols, m.coords))
    energies, e_tot, hlgap, t, _, _ = dft.jax_dft(s, args)
    g = golden("scf_oracle_ch4.npz")
    np.testing.assert_allclose(energies / 27.2114, g["energies"][:10, 0], atol=1e-6)
    e, energy, eigval, eigvec, dms, L_inv = dft.density_functional_theory(None, args)
    assert dms.shape == (10, 3, 9, 9)
    np.testing.assert_allclose(dms[:, 0], np.transpose(dms[:, 0], (0, 2, 1)), atol=1e-12)


def test_device_setup_matches_host(cuda):
    rng = np.random.default_rng(3)
    mols = [Mole(methane()), Mole(random_molecule(rng, 3)), Mole(random_molecule(rng, 5))]
    eng = RKSEngine(mols, level=0, precision="fp64")
    eng.device_setup()
    torch.cuda.synchronize()
    P = eng.plan
    off = P.grid_off
    coords = eng.coords.cpu().numpy().reshape(-1, 3)
    w = eng.weights.cpu().numpy()
    for mi, m in enumerate(mols):
        hs = HostSetup(m, 0)
        for name, ref in (("S", hs.S), ("T", hs.T), ("V", hs.V), ("Linv", hs.L_inv), ("D0", hs.D0)):
            got = P.unpack(getattr(eng, name).cpu().numpy(), mi)
            np.testing.assert_allclose(got, ref, atol=1e-10, err_msg=name)
        np.testing.assert_allclose(coords[off[mi]:off[mi + 1]], hs.coords, atol=1e-12)
        np.testing.assert_allclose(w[off[mi]:off[mi + 1]], hs.weights, rtol=1e-10, atol=1e-14)
        assert abs(eng.enuc[mi].item() - hs.E_nuc) < 1e-10
    eng.close()


def test_run_converged_batched_mixed_vs_plain(cuda):
    rng = np.random.default_rng(21)
    mols = [Mole(random_molecule(rng, int(k))) for k in (1, 2, 4, 6, 3, 9)]
    eng = RKSEngine(mols, level=0, precision="mixed")
    res = eng.run_converged(max_its=40)
    assert bool(res["converged"].all())
    E = res["energy"].cpu().numpy()
    for mi, m in enumerate(mols):
        e1 = RKSEngine([m], level=0, precision="fp64")
        r1 = e1.run_converged(graph=False)
        e1.close()
        assert abs(E[mi] - float(r1["energy"][0])) <= 1e-4          # |dE| <= 0.1 mHa
    eng.close()


def test_converged_graph_equals_eager(cuda):
    rng = np.random.default_rng(8)
    mols = [Mole(random_molecule(rng, 3)), Mole(methane())]
    a = RKSEngine(mols, level=0, precision="fp64").run_converged(graph=True)
    b = RKSEngine(mols, level=0, precision="fp64").run_converged(graph=False)
    np.testing.assert_allclose(a["energy"].cpu().numpy(), b["energy"].cpu().numpy(), atol=1e-10)
    assert (a["iterations"].cpu().numpy() == b["iterations"].cpu().numpy()).all()


def test_captured_iteration_reused_until_the_plan_changes(cuda):
    # a second run on the same engine replays the first run's graph; a knob change recaptures
    rng = np.random.default_rng(9)
    mols = [Mole(random_molecule(rng, k)) for k in (2, 5, 1)]
    eng = RKSEngine(mols, level=0, precision="mixed", tuned=False)
    a = eng.run_converged()
    g1 = eng._graph[1]
    eng._eri_done = False
    b = eng.run_converged()
    assert eng._graph[1] is g1
    eng.plan.set_xc_impl(1)
    c = eng.run_converged()
    assert eng._graph[1] is not g1
    for r in (b, c):
        np.testing.assert_allclose(r["energy"].cpu().numpy(), a["energy"].cpu().numpy(), atol=2e-6)
        assert (r["iterations"].cpu().numpy() == a["iterations"].cpu().numpy()).all()
    eng.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config2_level3_per_precision(cuda, precision):
    """the seeded 9-heavy-atom molecule (nao 62) on the level-3 grid (426 762 points), plain FP64
    and mixed precision against the FP64 oracle: J/K on the oracle's converged density and the
    energies of 20 iterations from the same guess (its ERIs: test_eri_config2_full)"""
    g = golden("scf_oracle_config2_level3.npz")
    m = Mole(str(g["atom"]), unit=str(g["unit"]))
    setup = HostSetup(m, 3)
    assert len(setup.weights) == int(g["npoints"])
    eng = RKSEngine([m], level=3, precision=precision, setups=[setup])
    try:
        res = eng.run(its=20, log=False)
        D = g["D"]
        eng.jk(D=torch.from_numpy(eng.plan.pack([D])).to(cuda))
        torch.cuda.synchronize()
        J = eng.plan.unpack(eng.J.cpu().numpy(), 0)
        K = eng.plan.unpack(eng.K.cpu().numpy(), 0)
    finally:
        eng.close()
    _, Jr, Kr = rks.jk_from_s8(D, oeri.eri_s8(m), m.nao)
    tol = 1e-9 if precision == "fp64" else 2e-5 * max(1.0, np.abs(Jr).max())
    np.testing.assert_allclose(J, Jr, atol=tol, rtol=0)
    np.testing.assert_allclose(K, Kr, atol=tol, rtol=0)
    E = res["energies"][:, 0, 0]
    if precision == "fp64":
        assert np.abs(E - g["energies"][:, 0]).max() <= 1e-6          # every iteration
    else:
        assert abs(E[-1] - g["energies"][-1, 0]) <= 1e-4              # north-star: 0.1 mHa


def test_nanodft_thresholds(cuda):
    """ao_threshold and eri_threshold (nanoDFT.py:221-230, 280-288) against the oracle SCF on the
    same thresholded AO values, grid and ERIs"""
    thr_ao, thr_eri = 1e-2, 1e-6
    opts, mol_str = nanodft.nanoDFT_options(its=12, mol_str="water", level=0, ao_threshold=thr_ao,
                                            eri_threshold=thr_eri)
    mol = nanodft.build_mol(mol_str, opts.basis)
    E, (logged, hl, mo_e, mo_c, coords, w) = nanodft.nanoDFT(mol, opts)
    s = HostSetup(mol, 0, ao_threshold=thr_ao)
    assert len(w) == len(s.weights) < len(HostSetup(mol, 0).weights)
    s8 = oeri.eri_s8(mol)
    s8[np.abs(s8) <= thr_eri] = 0.0
    ref = rks.scf(s.S, s.T, s.V, s.D0, s8, s.ao, s.weights, mol.nelectron // 2, s.E_nuc, its=12)
    np.testing.assert_allclose(E[:, 0] / HARTREE_TO_EV, ref["energies"][:, 0], atol=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_scf_iterate_entry_equals_individual_entries(cuda, precision):
    # b2_scf_iterate (one C call per SCF iteration, over a b2_scf_state struct) against the same
    # iteration made of the individual entry points, on an uneven batch with one molecule inactive
    rng = np.random.default_rng(21)
    mols = [Mole(random_molecule(rng, k)) for k in (1, 4, 2, 7)]
    out = {}
    keep = None
    for path in ("iterate", "entries"):
        eng = RKSEngine(mols, level=0, precision=precision, guess="minao")
        if keep is None:                        # matrix entries of the active molecules
            keep = np.concatenate([np.arange(eng.plan.mat_off[m], eng.plan.mat_off[m] + eng.plan.nao[m] ** 2)
                                   for m in (0, 1, 3)])
        eng.prepare()
        eng.initial()
        eng.active[2] = 0
        E = []
        for _ in range(6):
            (eng.step if path == "iterate" else eng.step_entries)()
            E.append(eng.energy.view(len(mols), 5).cpu().numpy().copy())
        torch.cuda.synchronize()
        out[path] = (np.array(E), eng.iter.cpu().numpy().copy(), eng.diffJK.cpu().numpy().copy())
        eng.close()
    Ei, it_i, dj_i = out["iterate"]
    Ee, it_e, dj_e = out["entries"]
    np.testing.assert_array_equal(it_i, [6, 6, 0, 6])
    np.testing.assert_array_equal(it_i, it_e)
    np.testing.assert_allclose(Ei, Ee, atol=1e-9, rtol=0)
    # the inactive molecule: b2_scf_iterate leaves its buffers untouched, the element-wise torch
    # op of the entry-point path rewrites its diff_JK; the active ones agree
    np.testing.assert_allclose(dj_i[keep], dj_e[keep], atol=1e-9, rtol=0)
