"""Drop-in for the DFT driver of pyscf_ipu/dft.py (what the README calls
density_functional_theory.py).

``density_functional_theory(atom_positions, args, mf_diis_space=9)`` (dft.py:197-747) reads
the module-level ``mol`` set by ``jax_dft`` (dft.py:1302-1347) and returns
``(e, energy, eigenvalues, eigenvectors, dms, L_inv)``: e = per-iteration total energy [Ha],
dms = (its, 3, N, N) holding [density matrix, J, Hamiltonian] per iteration (dft.py:866-875).
Two placeholders of the reference are filled with real values: ``energy`` is the final total
energy and ``eigenvalues`` the final orbital energies (the reference returns its zero-
initialised buffers, dft.py:95-96, 183-185).  ``eigenvectors`` is the occupied-masked MO
coefficient matrix as in dft.py:841-842.
"""
import argparse
import sys
import time
import numpy as np

from .constants import HARTREE_TO_EV, HYB_B3LYP
from .mole import Mole, methane
from .engine import RKSEngine, HostSetup

hartree_to_eV = 27.2114        # dft.py:47
mol = None


def get_args(argv=None):
    """The hot-path subset of dft.py's flags (dft.py:1349-1429)."""
    p = argparse.ArgumentParser(description="Arguments for Density Functional Theory (B200).")
    p.add_argument("-its", default=20, type=int, help="Number of Kohn-Sham iterations.")
    p.add_argument("-spin", default=0, type=int)
    p.add_argument("-str", default="", help='Molecule string, e.g., "H 0 0 0; H 0 0 1; O 1 0 0; " (Bohr)')
    p.add_argument("-float32", action="store_true", help="Mixed precision (FP32 ERI/JK/grid).")
    p.add_argument("-basis", default="STO-3G")
    p.add_argument("-xc", default="b3lyp")
    p.add_argument("-backend", default="b200")
    p.add_argument("-level", default=2, type=int, help="Grid level (default 2).")
    p.add_argument("-skipdiis", action="store_true")
    p.add_argument("-density_mixing", action="store_true")
    p.add_argument("-choleskycpu", action="store_true")
    p.add_argument("-methane", action="store_true")
    p.add_argument("-H", action="store_true")
    p.add_argument("-he", action="store_true")
    p.add_argument("-benchmark", action="store_true")
    return p.parse_args(argv)


def density_functional_theory(atom_positions, args, mf_diis_space=9):
    if mf_diis_space != 9:
        raise ValueError("the device DIIS ring holds 9 entries (as the reference's IPU path)")
    if args.xc.lower() != "b3lyp":
        raise ValueError("only B3LYP is supported")
    # the reference's timing switches that skip or randomise work (dft.py:127-133, 827) change
    # the results; they are refused rather than ignored
    for flag in ("skiperi", "randeri", "skipeigh", "float16"):
        if getattr(args, flag, False):
            raise ValueError(f"-{flag} (a timing switch that skips or randomises work) is not supported")
    if mol is None:
        raise RuntimeError("set b200dft.dft.mol (jax_dft does) before calling")
    setup = HostSetup(mol, level=args.level)
    eng = RKSEngine([mol], precision="mixed" if args.float32 else "fp64", setups=[setup])
    try:
        if getattr(args, "density_mixing", False):
            res = _run_mixing(eng, args.its, not args.skipdiis)
        else:
            res = eng.run(its=args.its, use_diis=not args.skipdiis, log=True)
    finally:
        eng.close()
    N = mol.nao
    its = args.its
    logs = res["logs"][:, :, :N * N].reshape(its, 4, N, N)
    dms = np.stack([logs[:, 0], logs[:, 3], logs[:, 2]], axis=1)
    e = res["energies"][:, 0, 0].copy()
    nocc = mol.nelectron // 2
    C = res["C"][:N * N].reshape(N, N)
    mask = np.zeros(N)
    mask[:nocc] = 1
    eigenvalues = res["mo_energy"][-1, 0, :N]
    return e, e[-1], eigenvalues, C * mask[None, :], dms, setup.L_inv


def _run_mixing(eng, its, use_diis):
    """dft.py:848-849: D <- (D_old + D)/2 once the DIIS ring is full (cycle > 9)."""
    import torch
    eng.prepare()
    eng.initial()
    nm = eng.plan.nmol
    E, mo, logs = [], [], []
    for i in range(its):
        old = eng.D.clone()
        eng.fock_diis(use_diis)
        eng.eigh_density()
        if i > 9:
            eng.D.copy_(0.5 * (old + eng.D))
        eng.xc()
        eng.jk()
        eng.diffJK.copy_(eng.diff_jk())
        eng.energies()
        eng.iter.add_(1)
        E.append(eng.energy.view(nm, 5).clone())
        mo.append(eng.mo_energy.view(nm, -1).clone())
        logs.append(torch.stack([eng.D.clone(), eng.diffJK.clone(), eng.H.clone(), eng.J.clone()]))
    return dict(energies=torch.stack(E).cpu().numpy(), mo_energy=torch.stack(mo).cpu().numpy(),
                logs=torch.stack(logs).cpu().numpy(), C=eng.C.cpu().numpy())


def jax_dft(str, args):
    """dft.py:1302-1347: build ``mol`` (Bohr), run, return (energies eV, e_tot, hlgap, t, t, hlgap)."""
    global mol
    mol = Mole(str, basis=args.basis, unit="Bohr", spin=args.spin)
    t0 = time.time()
    energies, e_tot, mo_energy, mo_coeff, dms, L_inv = density_functional_theory(mol.atom_coords(), args)
    t = time.time() - t0
    e_tot = energies[-1] * hartree_to_eV
    N = mol.nao
    nocc = mol.nelectron // 2
    mo_e = np.linalg.eigh(L_inv @ dms[-1, 2] @ L_inv.T)[0]
    hlgap = hartree_to_eV * abs(mo_e[nocc - 1] - mo_e[nocc])
    return energies * hartree_to_eV, e_tot, hlgap, t, t, hlgap


def main(argv=None):
    args = get_args(argv)
    if args.methane:
        from .constants import ANGSTROM_TO_BOHR
        m = Mole(methane())
        s = "; ".join(f"{sym} {x} {y} {z}" for sym, (x, y, z) in zip(m.symbols, m.coords))
    elif args.H:
        s = "H 0 0 0; H 0 0 1.4"
    elif args.he:
        raise SystemExit("He: odd shells are not in the STO-3G table here")
    else:
        s = args.str
    if not s:
        raise SystemExit("give -str '<atoms in Bohr>' or -methane")
    energies, e_tot, hlgap, t, _, _ = jax_dft(s, args)
    print(energies)
    print("E [eV] %.6f  HL gap [eV] %.6f  time %.3fs" % (e_tot, hlgap, t))
    return energies


if __name__ == "__main__":
    main()
