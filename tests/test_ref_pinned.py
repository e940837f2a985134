"""The oracle against fixtures made by the reference's OWN Python code (b3lyp, nanoDFT, the
sparse s8 J/K), run unmodified under a numpy stand-in for jax (tests/golden/make_ref_golden.py).

These pin the oracle's restatement of exchange_correlation/*.py, nanoDFT.py (iteration, DIIS,
pinv, energy, final eigh) and sparse_symmetric_ERI.py to the reference itself; the GPU tests
in test_gpu_ref_pinned.py compare the B200 kernels with the same fixtures.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import eri as oeri, rks
from b200dft.constants import HARTREE_TO_EV
from b200dft.mole import Mole
from b200dft.int1e import int1e
from b200dft.grids import build_grid
from b200dft.guess import minao

NAMES = ("ch4", "water", "tree3")


def test_b3lyp_oracle_equals_reference():
    g = golden("ref_b3lyp.npz")
    e, vr, vg = rks.b3lyp(g["rho"], float(g["eps"]))
    np.testing.assert_allclose(e, g["exc"], rtol=1e-11, atol=0)
    np.testing.assert_allclose(vr, g["vrho"], rtol=1e-11, atol=0)
    np.testing.assert_allclose(vg, g["vgamma"], rtol=1e-11, atol=1e-300)


def setup_inputs(name):
    """the molecule and the setup arrays the fixture was made from; checks that they did not
    drift since (grid size and weight sum, overlap and guess sums)"""
    f = golden(f"ref_nanodft_{name}.npz")
    m = Mole(str(f["atom"]))
    g = build_grid(m, int(f["level"]))
    S, T, V = int1e(m)
    D0 = minao(m)
    assert len(g.weights) == int(f["n_points"])
    assert abs(g.weights.sum() - float(f["weight_sum"])) <= 1e-9 * abs(float(f["weight_sum"]))
    assert abs(S.sum() - float(f["S_sum"])) <= 1e-12 * abs(float(f["S_sum"]))
    assert abs(D0.sum() - float(f["D0_sum"])) <= 1e-12 * max(1.0, abs(float(f["D0_sum"])))
    return f, m, g, S, T, V, D0


@pytest.mark.parametrize("name", NAMES)
def test_scf_oracle_equals_reference_nanodft(name):
    f, m, g, S, T, V, D0 = setup_inputs(name)
    r = rks.scf(S, T, V, D0, oeri.ref_eri_s8(m) if oeri.ref_available() else oeri.eri_s8(m),
                rks.ao_values(m, g.coords), g.weights, m.nelectron // 2, m.energy_nuc(), its=int(f["its"]))
    # every iteration's five energy terms, the final orbital energies (Hartree)
    np.testing.assert_allclose(r["energies"], f["energies"] / HARTREE_TO_EV, atol=1e-9, rtol=0)
    np.testing.assert_allclose(r["energies"], f["logged"] / HARTREE_TO_EV, atol=1e-9, rtol=0)
    np.testing.assert_allclose(r["mo_energy"], f["mo_energy"], atol=1e-9, rtol=0)


@pytest.mark.parametrize("name", NAMES)
def test_s8_jk_oracle_equals_reference_sparse_einsum(name):
    f = golden(f"ref_sparse_jk_{name}.npz")
    m = Mole(str(f["atom"]))
    s8 = oeri.ref_eri_s8(m) if oeri.ref_available() else oeri.eri_s8(m)
    djk = rks.jk_from_s8(f["D"], s8, m.nao)[0]
    np.testing.assert_allclose(djk, f["diff_JK"], atol=1e-12, rtol=0)
