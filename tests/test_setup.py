"""Host setup: basis, molecule, grids, generator, 1e integrals (CPU)."""
import numpy as np

from b200dft.mole import Mole, methane
from b200dft import grids
from b200dft.molgen import config2_molecule, config3_batch, random_molecule
from b200dft.int1e import int1e
from b200dft.guess import minao


def test_lebedev_exactness():
    for n, deg in ((26, 7), (50, 11), (86, 15)):
        p, w = grids.lebedev(n)
        assert len(p) == n and abs(w.sum() - 1) < 1e-14
        np.testing.assert_allclose((p * p).sum(1), 1, atol=1e-14)
        for a in range(deg // 2 + 1):
            for b in range(deg // 2 + 1 - a):
                c = 0
                val = (w * p[:, 0] ** (2 * a) * p[:, 1] ** (2 * b)).sum()
                assert abs(val - grids._sphere_moment(a, b, c)) < 1e-13


def test_product_rule_exactness():
    p, w = grids.product_rule(29)
    for a, b, c in ((7, 7, 0), (3, 4, 7), (0, 0, 14)):
        val = (w * p[:, 0] ** (2 * a) * p[:, 1] ** (2 * b) * p[:, 2] ** (2 * c)).sum()
        assert abs(val - grids._sphere_moment(a, b, c)) < 1e-13


def test_grid_integrates_density():
    m = Mole(methane())
    g = grids.build_grid(m, 0)
    S, T, V = int1e(m)
    from oracle import rks
    ao = rks.ao_values(m, g.coords)
    D = minao(m)
    n = ((ao[0] @ D) * ao[0]).sum(1) @ g.weights
    assert abs(n - np.trace(D @ S)) < 2e-2          # level-0 grid: electrons to ~1e-3 relative
    assert g.weights.min() >= 0


def test_becke_partition_of_unity():
    m = Mole("C 0 0 0; O 0 0 1.2; H 0.9 0.5 -0.3; H -0.9 0.5 -0.3")
    c = np.random.default_rng(0).normal(size=(500, 3)) * 2
    p = grids.becke_partition(c, m.atom_coords(), m.atom_charges())
    np.testing.assert_allclose(p.sum(0), 1, atol=1e-12)


def test_mole_layout():
    m = Mole(methane())
    assert m.nao == 9 and m.nelectron == 10 and m.nbas == 7
    assert list(m.ao_loc) == [0, 1, 2, 5, 6, 7, 8, 9]
    S, T, V = int1e(m)
    np.testing.assert_allclose(np.diag(S), 1, atol=1e-12)
    assert np.linalg.eigvalsh(S).min() > 0
    np.testing.assert_allclose(S, S.T, atol=1e-14)
    np.testing.assert_allclose(T, T.T, atol=1e-12)
    np.testing.assert_allclose(V, V.T, atol=1e-12)
    D = minao(m)
    assert abs(np.trace(D @ S) - m.nelectron) < 1e-12


def test_generator_properties():
    s = config2_molecule(0)
    m = Mole(s)
    heavy = [x for x in m.symbols if x != "H"]
    assert len(heavy) == 9 and set(heavy) <= {"C", "N", "O"}
    assert m.nao <= 65 and m.nelectron % 2 == 0
    d = np.sqrt(((m.coords[:, None] - m.coords[None]) ** 2).sum(-1)) * 0.52917721092
    np.fill_diagonal(d, 9)
    assert d.min() > 0.89
    b = config3_batch(64, seed=3)
    assert config3_batch(64, seed=3) == b                 # seeded
    nao = [Mole(x).nao for x in b]
    assert 5 <= min(nao) and max(nao) <= 65


def test_kinetic_fd_identity():
    # T = -1/2 <a|lap|b>; symmetric and positive definite
    m = Mole("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7572 -0.4692")
    S, T, V = int1e(m)
    assert np.linalg.eigvalsh(T).min() > 0


def test_host_ao_values_match_oracle():
    from oracle import rks
    from b200dft.ao import eval_ao
    m = Mole("N 0 0 0; C 0 0 2.6; O 2.1 0 3.9; H 0 1.9 -0.8", unit="Bohr")
    g = grids.Grids(m, 0).build()
    a = eval_ao(m, g.coords)
    np.testing.assert_allclose(a, rks.ao_values(m, g.coords), atol=1e-13, rtol=0)


def test_ao_threshold_as_nanodft():
    """b200dft.ao.threshold_grid against the reference's steps, nanoDFT.py:221-230, written out"""
    from oracle import rks
    from b200dft.ao import threshold_grid
    m = Mole(methane())
    g = grids.Grids(m, 0).build()
    coords, w = np.asarray(g.coords), np.asarray(g.weights)
    ao = rks.ao_values(m, coords)
    for thr in (1e-6, 1e-3, 1e-2):
        A = ao.copy()
        A[np.abs(A) < thr] = 0
        sparsity_mask = np.where(np.all(A == 0, axis=0), 0, 1)
        sparse_rows = np.where(np.all(sparsity_mask == 0, axis=1), 0, 1).reshape(-1, 1)
        drop = np.where(sparse_rows == 0)[0]
        ref = (np.delete(A, drop, axis=1), np.delete(coords, drop, axis=0), np.delete(w, drop, axis=0))
        got = threshold_grid(ao, coords, w, thr)
        for x, y in zip(got, ref):
            np.testing.assert_array_equal(x, y)
    assert len(got[2]) < len(w)                  # the largest threshold drops points


def test_host_setup_with_ao_threshold():
    from b200dft.engine import HostSetup
    m = Mole(methane())
    s0 = HostSetup(m, level=0)
    s1 = HostSetup(m, level=0, ao_threshold=1e-2)
    assert s0.ao is None and s1.ao.shape == (4, len(s1.weights), m.nao)
    assert 0 < len(s1.weights) < len(s0.weights) and s1.coords.shape == (len(s1.weights), 3)


def test_dft_dropin_refuses_work_skipping_switches():
    import types
    import pytest
    from b200dft import dft
    for flag in ("skiperi", "randeri", "skipeigh", "float16"):
        args = types.SimpleNamespace(xc="b3lyp", its=2, level=0, float32=False, skipdiis=False, **{flag: True})
        with pytest.raises(ValueError, match=flag):
            dft.density_functional_theory(None, args)


def test_double_factorial_known_values():
    # the reference's known answers for factorial2 (test/test_special.py:27-34); the grid's
    # sphere moments are built from this function
    from b200dft.grids import _dfact
    assert [_dfact(n) for n in range(1, 9)] == [1, 2, 3, 8, 15, 48, 105, 384]
    assert _dfact(0) == 1 and _dfact(-1) == 1
