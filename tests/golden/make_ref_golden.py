"""Golden fixtures produced by running the reference's OWN Python code (unmodified, imported
from the reference checkout) under the numpy stand-in of ``ref_standin.py``.

    python oracle/build_ref.py && python tests/golden/make_ref_golden.py

The reference checkout is taken from $PYSCF_IPU_REFERENCE (default /root/reference); it is
read here only, never by the tests, ``smoke()`` or ``bench.py``.

* ref_b3lyp.npz: ``b3lyp(rho, EPSILON_B3LYP)`` (pyscf_ipu/exchange_correlation/b3lyp.py:13-39,
  with lda.py, vwn.py, b88.py, lyp.py) on a seeded sweep of densities and gradients that spans
  the clip limits (rho0 from 1e-12 to 1e3, |grad rho| from 0 to ~1e3).
* ref_nanodft_<name>.npz: the reference driver ``nanoDFT(mol, opts)``
  (pyscf_ipu/nanoDFT/nanoDFT.py:259-336: its setup, ``_nanoDFT``, 20 x ``nanoDFT_iteration``
  with DIIS, ``exchange_correlation``, dense ``get_JK``, ``energy``, ``hlgap``, final eigh) in
  float64 with the dense ERI tensor, for molecules whose PySCF-side inputs (grid, AO values,
  one-electron matrices, guess) come from this project's setup code (PySCF is absent) and whose
  ERIs come from the reference's compiled ``int2e_sph`` (oracle/_ref).  Stored: energies and
  logged energies (its, 5) in eV, hlgaps, final mo_energy, and checksums of the inputs.
* ref_sparse_jk_<name>.npz: ``sparse_symmetric_einsum`` (pyscf_ipu/nanoDFT/
  sparse_symmetric_ERI.py:86-137, backend "cpu") on the s8 list packed as nanoDFT packs it
  (nanoDFT.py:283-315: nonzero entries divided by ``num_repetitions_fast``, (i,j,k,l) as int16
  bit-cast to float16), float64 values, for a seeded symmetric density; stored: diff_JK.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("PYSCF_IPU_REFERENCE", "/root/reference")
sys.path.insert(0, os.path.join(ROOT, "pyscf-ipu_b200"))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import ref_standin                                              # noqa: E402

MOLS = {
    "ch4": None,        # filled in main() (needs b200dft)
    "water": "O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7572 -0.4692",
    "tree3": None,
}


def b3lyp_sweep(n=4000, seed=11):
    """rho (4, n): rho0 log-uniform over [1e-12, 1e3] (below and above the clip at 1e-9),
    half-gradients with |.| log-uniform over [1e-12, 1e3] in random directions, plus exact
    zeros of the gradient"""
    rng = np.random.default_rng(seed)
    rho = np.zeros((4, n))
    rho[0] = 10.0 ** rng.uniform(-12, 3, n)
    d = rng.normal(size=(3, n))
    d /= np.linalg.norm(d, axis=0)
    g = 10.0 ** rng.uniform(-12, 3, n)
    g[: n // 20] = 0.0
    rho[1:4] = d * g
    return rho


def main():
    sys.path.insert(0, REF)
    ref_standin.install()
    from pyscf_ipu.exchange_correlation.b3lyp import b3lyp
    import pyscf_ipu.nanoDFT.nanoDFT                            # noqa: F401
    import pyscf_ipu.nanoDFT.sparse_symmetric_ERI               # noqa: F401
    # the package's __init__ re-exports the function nanoDFT under the module's name
    rn = sys.modules["pyscf_ipu.nanoDFT.nanoDFT"]
    rs = sys.modules["pyscf_ipu.nanoDFT.sparse_symmetric_ERI"]

    from oracle import eri as oeri, rks
    from b200dft.mole import Mole, methane
    from b200dft.molgen import random_molecule
    from b200dft.int1e import int1e
    from b200dft.grids import build_grid
    from b200dft.guess import minao
    assert oeri.ref_available(), "build oracle/_ref first (python oracle/build_ref.py)"

    rho = b3lyp_sweep()
    e, vr, vg = b3lyp(rho, rn.EPSILON_B3LYP)
    np.savez_compressed(os.path.join(HERE, "ref_b3lyp.npz"), rho=rho, exc=np.asarray(e), vrho=np.asarray(vr),
                        vgamma=np.asarray(vg), eps=rn.EPSILON_B3LYP)
    print("b3lyp", len(e))

    MOLS["ch4"] = methane()
    MOLS["tree3"] = random_molecule(np.random.default_rng(7), 3)

    def grid(m, level):
        g = build_grid(m, level)
        return g.coords, g.weights

    for name, atom in MOLS.items():
        m = Mole(atom)
        fm = ref_standin.FakeMol(m, grid, rks.ao_values, int1e, minao, oeri.ref_eri_s8, oeri.unpack_s8)
        from collections import namedtuple
        fields = dict(its=20, float32=False, basis="sto-3g", xc="b3lyp", backend="cpu", level=0, diis=True,
                      structure_optimization=False, eri_threshold=0.0, ao_threshold=0.0, batches=1,
                      ndevices=1, dense_ERI=True, v=False, profile=False, vis_num_error=False,
                      molecule_name=name)
        opts = namedtuple("DFTOptionsImmutable", fields.keys())(**fields)
        energies, (logged, hlgaps, mo_energy, mo_coeff, coords, weights) = rn.nanoDFT(fm, opts)
        S, T, V = int1e(m)
        np.savez_compressed(os.path.join(HERE, f"ref_nanodft_{name}.npz"), energies=np.asarray(energies),
                            logged=np.asarray(logged), hlgaps=np.asarray(hlgaps),
                            mo_energy=np.asarray(mo_energy), atom=atom, level=0, its=20,
                            n_points=len(weights), weight_sum=float(np.sum(weights)),
                            S_sum=float(S.sum()), D0_sum=float(minao(m).sum()))
        print(name, m.nao, len(weights), energies[-1, 0] / rn.HARTREE_TO_EV)

        # sparse s8 J/K (packing as nanoDFT.py:283-315, float64 values, one batch, one device)
        s8 = oeri.ref_eri_s8(m)
        nz = np.nonzero(s8)[0].astype(np.uint64)
        ij, kl = rs.get_i_j(nz)
        rep = rs.num_repetitions_fast(ij, kl)
        vals = s8[nz] / rep
        i, j = rs.get_i_j(ij)
        k, l = rs.get_i_j(kl)
        idx = np.vstack([i, j, k, l]).T.reshape(1, -1, 4).astype(np.int16).view(np.float16)
        rng = np.random.default_rng(5)
        A = rng.normal(size=(m.nao, m.nao))
        D = (A + A.T) / 2
        djk = np.asarray(rs.sparse_symmetric_einsum(vals.reshape(1, -1), idx, D, "cpu")).reshape(m.nao, m.nao)
        np.savez_compressed(os.path.join(HERE, f"ref_sparse_jk_{name}.npz"), D=D, diff_JK=djk, atom=atom)
        print(name, "sparse J/K", len(vals))


if __name__ == "__main__":
    main()
