"""Generate the golden fixtures in this directory (run where the reference is available).

    python oracle/build_ref.py && make -C oracle ref && python tests/golden/make_golden.py

* eri_ref_<name>.npz: s8 ERIs computed by the reference's OWN compiled FP64 libcint port
  (``int2e_sph``, pyscf_ipu/electron_repulsion/cpu_int2e_sph.cpp:7706, built from the
  reference sources by oracle/build_ref.py) for small molecules, with the molecule string.
* eri_ref_sample_config2.npz: for the seeded 9-heavy-atom molecule (too large to store in
  full) the reference's values at 4096 seeded positions plus sum and sum of squares.
* scf_oracle_<name>.npz: FP64 oracle SCF trajectory (energies per iteration, final
  mo_energy) on this project's level-0 grid; used to pin later changes of the oracle.
* scf_oracle_config2_level3.npz: the same for the seeded 9-heavy-atom molecule on the level-3
  grid (426 762 points), plus the final density, for the single-molecule precision comparison.
"""
import os
import sys
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pyscf-ipu_b200"))
sys.path.insert(0, ROOT)

from oracle import eri, rks                         # noqa: E402
from b200dft.mole import Mole, methane              # noqa: E402
from b200dft.molgen import config2_molecule, random_molecule  # noqa: E402
from b200dft.int1e import int1e                     # noqa: E402
from b200dft.grids import build_grid                # noqa: E402
from b200dft.guess import minao                     # noqa: E402

MOLS = {
    "h2": ("H 0 0 0; H 1.4 0 0", "Bohr"),
    "ch4": (methane(), "Angstrom"),
    "water": ("O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7572 -0.4692", "Angstrom"),
    "tree3": (random_molecule(np.random.default_rng(7), 3), "Angstrom"),
}


def main():
    for name, (s, unit) in MOLS.items():
        m = Mole(s, unit=unit)
        v = eri.ref_eri_s8(m)
        np.savez_compressed(os.path.join(HERE, f"eri_ref_{name}.npz"), s8=v, atom=s, unit=unit)
        print(name, m, len(v))
    m = Mole(config2_molecule(0))
    v = eri.ref_eri_s8(m)
    rng = np.random.default_rng(123)
    idx = np.sort(rng.choice(len(v), 4096, replace=False))
    np.savez_compressed(os.path.join(HERE, "eri_ref_sample_config2.npz"), idx=idx, val=v[idx],
                        total=v.sum(), sumsq=(v * v).sum(), atom=config2_molecule(0), n=len(v))
    print("config2", m, len(v))
    for name in ("ch4", "water"):
        s, unit = MOLS[name]
        m = Mole(s, unit=unit)
        g = build_grid(m, 0)
        S, T, V = int1e(m)
        ao = rks.ao_values(m, g.coords)
        r = rks.scf(S, T, V, minao(m), eri.ref_eri_s8(m), ao, g.weights, m.nelectron // 2,
                    m.energy_nuc(), its=20)
        np.savez_compressed(os.path.join(HERE, f"scf_oracle_{name}.npz"), energies=r["energies"],
                            mo_energy=r["mo_energy"], atom=s, unit=unit, level=0)
        print(name, r["energies"][-1, 0])
    scf_config2_level3()


def scf_config2_level3():
    m = Mole(config2_molecule(0))
    g = build_grid(m, 3)
    S, T, V = int1e(m)
    ao = rks.ao_values(m, g.coords)
    r = rks.scf(S, T, V, minao(m), eri.ref_eri_s8(m), ao, g.weights, m.nelectron // 2, m.energy_nuc(),
                its=20)
    np.savez_compressed(os.path.join(HERE, "scf_oracle_config2_level3.npz"), energies=r["energies"],
                        mo_energy=r["mo_energy"], D=r["logs"][-1, 0], atom=config2_molecule(0),
                        unit="Angstrom", level=3, npoints=len(g.weights))
    print("config2 level 3", r["energies"][-1, 0], len(g.weights))


if __name__ == "__main__":
    main()
