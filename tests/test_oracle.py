"""The oracle itself, pinned against the reference's own numbers (CPU)."""
import numpy as np
import pytest

from conftest import golden
from oracle import eri, rks
from b200dft.mole import Mole, methane
from b200dft.int1e import int1e
from b200dft.grids import build_grid
from b200dft.guess import minao


def test_eri_oracle_vs_reference_golden():
    # golden s8 lists were produced by the reference's compiled int2e_sph (make_golden.py)
    for name in ("h2", "ch4", "water", "tree3"):
        g = golden(f"eri_ref_{name}.npz")
        m = Mole(str(g["atom"]), unit=str(g["unit"]))
        np.testing.assert_allclose(eri.eri_s8(m), g["s8"], atol=1e-12, rtol=0)


def test_eri_oracle_config2_sample():
    g = golden("eri_ref_sample_config2.npz")
    m = Mole(str(g["atom"]))
    assert eri.n_s8(m.nao) == int(g["n"])
    # known values of the full-size molecule without recomputing everything: shell-free check
    # through the checksum of the whole list is done in the GPU suite; here 64 sampled shells
    v = eri.eri_s8(m)
    np.testing.assert_allclose(v[g["idx"]], g["val"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(v.sum(), float(g["total"]), rtol=1e-12)


def test_known_answers_h2_sto3g():
    # Szabo & Ostlund eq. 3.235, pinned in the reference at test/test_integrals.py:121-133
    m = Mole("H 0 0 0; H 1.4 0 0", unit="Bohr")
    E = eri.unpack_s8(eri.eri_s8(m), 2)
    assert abs(E[0, 0, 0, 0] - 0.7746) < 1e-4
    assert abs(E[0, 0, 1, 1] - 0.5697) < 1e-4
    assert abs(E[1, 0, 0, 0] - 0.4441) < 1e-4
    assert abs(E[1, 0, 1, 0] - 0.2970) < 1e-4
    S, T, V = int1e(m)
    # test_integrals.py:56-60 (kinetic) and 93-99 (nuclear, summed over the two centres)
    np.testing.assert_allclose(T, [[0.7600, 0.2365], [0.2365, 0.7600]], atol=1e-4)
    np.testing.assert_allclose(V, [[-1.2266 - 0.6538, -2 * 0.5974], [-2 * 0.5974, -1.2266 - 0.6538]],
                               atol=1e-4)
    assert abs(S[0, 1] - 0.6593) < 1e-4


def test_known_answers_primitives():
    # test_integrals.py:113-117: (ss|ss) = 2/sqrt(pi) and (ss|pxpx) = 0.940316 for unit
    # normalised alpha=1 primitives at the origin; built as single-primitive shells
    s = "H 0 0 0; H 0 0 0"
    m = Mole(s, unit="Bohr")
    # replace the basis with one normalised primitive of exponent 1
    from b200dft.basis import normalized_coefficients
    env = m._env.copy()
    for sh in range(m.nbas):
        m._bas[sh, 2] = 1
        env[m._bas[sh, 5]] = 1.0
        env[m._bas[sh, 6]] = normalized_coefficients(0, [1.0], [1.0])[0]
    m._env = env
    v = eri.eri_s8(m)
    assert abs(v[0] - 2 / np.sqrt(np.pi)) < 1e-12
    if eri.ref_available():
        assert abs(eri.ref_eri_s8(m)[0] - 2 / np.sqrt(np.pi)) < 1e-12


def test_boys_oracle():
    from scipy.special import gammainc, gamma
    for t in (1e-8, 0.3, 2.0, 11.0, 39.0, 41.0, 90.0):
        f = eri.boys(4, t)
        for mm in range(5):
            a = mm + 0.5
            ref = gamma(a) * gammainc(a, t) / (2 * t ** a)
            assert abs(f[mm] - ref) < 1e-14 * max(1, ref) + 1e-15


def test_b3lyp_oracle_derivatives_fd():
    rng = np.random.default_rng(0)
    rho = np.zeros((4, 64))
    rho[0] = 10 ** rng.uniform(-4, 1, 64)
    rho[1:] = rng.normal(size=(3, 64)) * rho[0] * 0.5
    e, vr, vg = rks.b3lyp(rho)
    # energy density per volume: rho0 * e_xc; check d/drho by central differences
    h = 1e-6 * rho[0]
    rp, rm = rho.copy(), rho.copy()
    rp[0] += h
    rm[0] -= h
    fd = ((rp[0] * rks.b3lyp(rp)[0]) - (rm[0] * rks.b3lyp(rm)[0])) / (2 * h)
    np.testing.assert_allclose(vr, fd, rtol=1e-6)


def test_scf_oracle_golden():
    for name in ("ch4", "water"):
        g = golden(f"scf_oracle_{name}.npz")
        m = Mole(str(g["atom"]), unit=str(g["unit"]))
        grid = build_grid(m, int(g["level"]))
        S, T, V = int1e(m)
        ao = rks.ao_values(m, grid.coords)
        r = rks.scf(S, T, V, minao(m), eri.eri_s8(m), ao, grid.weights, m.nelectron // 2,
                    m.energy_nuc(), its=20)
        np.testing.assert_allclose(r["energies"], g["energies"], atol=1e-9)


def test_ao_values_fd():
    m = Mole(methane())
    c = np.random.default_rng(1).normal(size=(20, 3))
    a = rks.ao_values(m, c)
    h = 1e-5
    for k in range(3):
        cp, cm = c.copy(), c.copy()
        cp[:, k] += h
        cm[:, k] -= h
        fd = (rks.ao_values(m, cp)[0] - rks.ao_values(m, cm)[0]) / (2 * h)
        np.testing.assert_allclose(a[1 + k], fd, atol=1e-6)
