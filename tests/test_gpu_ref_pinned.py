"""B200 kernels against fixtures made by the reference's OWN Python code (b3lyp, nanoDFT and
the sparse s8 J/K, run unmodified under a numpy stand-in for jax; tests/golden/
make_ref_golden.py): b2_b3lyp, the nanoDFT drop-in (float64 engine) and b2_jk_s8 /
b2_jk_pairs through the C ABI."""
import numpy as np
import pytest
import torch

from conftest import golden
from b200dft import nanodft
from b200dft.constants import HARTREE_TO_EV
from b200dft.engine import Plan
from b200dft.mole import Mole
from b200dft._lib import lib, check, ptr, stream_handle

pytestmark = pytest.mark.gpu

NAMES = ("ch4", "water", "tree3")


def test_b3lyp_entry_vs_reference(cuda):
    g = golden("ref_b3lyp.npz")
    rho = g["rho"]
    n = rho.shape[1]
    r = torch.from_numpy(np.ascontiguousarray(rho)).to(cuda)
    e, vr, vg = (torch.zeros(n, dtype=torch.float64, device=cuda) for _ in range(3))
    check(lib().b2_b3lyp(n, ptr(r), ptr(e), ptr(vr), ptr(vg), stream_handle()), "b2_b3lyp")
    torch.cuda.synchronize()
    np.testing.assert_allclose(e.cpu().numpy(), g["exc"], rtol=1e-11)
    np.testing.assert_allclose(vr.cpu().numpy(), g["vrho"], rtol=1e-11)
    np.testing.assert_allclose(vg.cpu().numpy(), g["vgamma"], rtol=1e-10)


@pytest.mark.parametrize("name", NAMES)
def test_nanodft_dropin_vs_reference_nanodft(cuda, name):
    # same molecule, same options (20 iterations, DIIS, level-0 grid, float64): the reference's
    # nanoDFT and this drop-in agree per iteration within 1e-6 Ha
    f = golden(f"ref_nanodft_{name}.npz")
    opts, mol_str = nanodft.nanoDFT_options(its=int(f["its"]), mol_str=str(f["atom"]), level=int(f["level"]))
    mol = nanodft.build_mol(mol_str, opts.basis)
    E, (logged, hl, mo_e, mo_c, coords, w) = nanodft.nanoDFT(mol, opts)
    assert len(w) == int(f["n_points"])
    tol = 1e-6 * HARTREE_TO_EV
    np.testing.assert_allclose(E, f["energies"], atol=tol, rtol=0)
    np.testing.assert_allclose(logged, f["logged"], atol=tol, rtol=0)
    np.testing.assert_allclose(hl, f["hlgaps"], atol=tol, rtol=0)
    np.testing.assert_allclose(mo_e, f["mo_energy"], atol=1e-6, rtol=0)


@pytest.mark.parametrize("entry", ["s8", "pairs"])
def test_jk_vs_reference_sparse_einsum(cuda, entry):
    fs = [golden(f"ref_sparse_jk_{n}.npz") for n in NAMES]
    mols = [Mole(str(f["atom"])) for f in fs]
    P = Plan(mols)
    eri = torch.full((P.n_eri,), float("nan"), dtype=torch.float64, device=cuda)
    check(lib().b2_eri_s8(P.h, 64, ptr(eri), stream_handle()), "b2_eri_s8")
    D = torch.from_numpy(P.pack([f["D"] for f in fs])).to(cuda)
    J = torch.zeros(P.n_mat, dtype=torch.float64, device=cuda)
    K = torch.zeros_like(J)
    if entry == "s8":
        check(lib().b2_jk_s8(P.h, 64, None, ptr(eri), ptr(D), ptr(J), ptr(K), stream_handle()), "b2_jk_s8")
    else:
        exch = torch.empty_like(eri)
        check(lib().b2_jk_exchange(P.h, 64, ptr(eri), ptr(exch), stream_handle()), "b2_jk_exchange")
        check(lib().b2_jk_pairs(P.h, 64, None, ptr(eri), ptr(exch), ptr(D), ptr(J), ptr(K), stream_handle()),
              "b2_jk_pairs")
    torch.cuda.synchronize()
    Jh, Kh = J.cpu().numpy(), K.cpu().numpy()
    for mi, f in enumerate(fs):
        djk = P.unpack(Jh, mi) - 0.1 * P.unpack(Kh, mi)        # diff_JK = J - K * hyb / 2
        np.testing.assert_allclose(djk, f["diff_JK"], atol=1e-10, rtol=0)
    P.close()
