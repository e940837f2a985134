"""Drop-in for nanoDFT's SCF entry (pyscf_ipu/nanoDFT/nanoDFT.py).

``nanoDFT(mol, opts)`` (nanoDFT.py:259-336) with ``opts = nanoDFT_options(...)``
(nanoDFT.py:548-618) returns ``(energies, (logged_energies, hlgaps, mo_energy, mo_coeff,
grid_coords, grid_weights))`` with energies (its, 5) in eV [E, E_core, E_J_K, E_xc, E_nuc].
The SCF runs on the B200 through the C ABI; ``float32=True`` selects the mixed-precision
form (FP32 ERIs, J/K and grid path; FP64 Fock, DIIS, eigensolve and energies).
"""
from collections import namedtuple
import numpy as np

from .constants import HARTREE_TO_EV, HYB_B3LYP, EPSILON_B3LYP
from .mole import Mole, build_mol, methane
from .grids import Grids
from .engine import RKSEngine, HostSetup

__all__ = ["nanoDFT", "nanoDFT_options", "build_mol", "energy", "hlgap", "process_mol_str", "grad"]

NAMED = {
    "methane": methane(),
    "h2": "H 0 0 0; H 0 0 0.74",
    "water": "O 0 0 0.1173; H 0 0.7572 -0.4692; H 0 -0.7572 -0.4692",
    "benzene": "; ".join(
        [f"C {1.39 * np.cos(a):.6f} {1.39 * np.sin(a):.6f} 0" for a in np.arange(6) * np.pi / 3] +
        [f"H {2.47 * np.cos(a):.6f} {2.47 * np.sin(a):.6f} 0" for a in np.arange(6) * np.pi / 3]),
}


def process_mol_str(mol_str):
    """Named molecule or an explicit atom string (nanoDFT utils.process_mol_str)."""
    return NAMED.get(mol_str.lower(), mol_str) if isinstance(mol_str, str) else mol_str


def energy(density_matrix, H_core, diff_JK, E_xc, E_nuc, _np=np):
    """nanoDFT.py:20-38."""
    E_core = _np.sum(density_matrix * H_core)
    E_J_K = _np.sum(density_matrix * diff_JK)
    E = E_core + E_J_K / 2 + E_xc + E_nuc
    return _np.array([E, E_core, E_J_K / 2, E_xc, E_nuc])


def hlgap(L_inv, H, n_electrons_half, _np=np):
    """nanoDFT.py:366-368."""
    mo_energy = _np.linalg.eigh(L_inv @ H @ L_inv.T)[0]
    return _np.abs(mo_energy[n_electrons_half] - mo_energy[n_electrons_half - 1])


def nanoDFT_options(its: int = 20, mol_str: str = "benzene", float32: bool = False,
                    basis: str = "sto-3g", xc: str = "b3lyp", backend: str = "b200", level: int = 0,
                    multv: int = 2, intv: int = 1, threads: int = 1, threads_int: int = 1,
                    diis: bool = True, structure_optimization: bool = False,
                    eri_threshold: float = 0.0, ao_threshold: float = 0.0, batches: int = 32,
                    ndevices: int = 1, dense_ERI: bool = False, v: bool = False,
                    profile: bool = False, vis_num_error: bool = False, molecule_name: str = None):
    """Same fields as the reference's nanoDFT_options (nanoDFT.py:548-618); returns
    (immutable options, processed mol_str).  its, float32, level, diis, eri_threshold and
    ao_threshold shape the B200 run; the IPU scheduling knobs (multv, intv, threads,
    threads_int, batches, ndevices) and dense_ERI (the dense and s8 ERI forms give the same J/K)
    leave it unchanged, and v / profile / vis_num_error (plots) are accepted and unused."""
    if xc.lower() != "b3lyp":
        raise ValueError("only B3LYP is supported (as in the reference, nanoDFT.py:627)")
    if molecule_name is None:
        molecule_name = mol_str
    mol_str = process_mol_str(mol_str)
    args = dict(locals())
    del args["mol_str"]
    Opts = namedtuple("DFTOptionsImmutable", list(args.keys()))
    return Opts(**args), mol_str


def nanoDFT(mol, opts):
    """Run the SCF for ``mol`` on the B200 (nanoDFT.py:259-336)."""
    if opts.structure_optimization:
        raise NotImplementedError("structure optimisation is outside the SCF hot path")
    # ao_threshold > 0: AO values below it are zeroed and grid points left without any are
    # dropped (nanoDFT.py:221-230); the SCF then reads those stored AO values
    setup = HostSetup(mol, level=opts.level, ao_threshold=opts.ao_threshold or 0.0)
    # eri_threshold > 0: s8 entries with |v| <= it are zeroed before J/K (nanoDFT.py:280-288)
    eng = RKSEngine([mol], precision="mixed" if opts.float32 else "fp64", setups=[setup],
                    eri_threshold=opts.eri_threshold or 0.0)
    try:
        res = eng.run(its=opts.its, use_diis=opts.diis, log=True)
    finally:
        eng.close()
    N = mol.nao
    its = opts.its
    logs = res["logs"][:, :, :N * N].reshape(its, 4, N, N)
    D, diffJK, H = logs[:, 0], logs[:, 1], logs[:, 2]
    logged = res["energies"][:, 0, :]
    nocc = mol.nelectron // 2
    energies = np.zeros((its, 5))
    hlgaps = np.zeros(its)
    for i in range(its):
        energies[i] = energy(D[i], setup.Hcore, diffJK[i], logged[i, 3], setup.E_nuc)
        mo_i = res["mo_energy"][i, 0, :N]
        hlgaps[i] = abs(mo_i[nocc] - mo_i[nocc - 1])
    mo_energy = res["mo_energy"][-1, 0, :N]
    mo_coeff = res["C"][:N * N].reshape(N, N)
    energies, logged, hlgaps = [a * HARTREE_TO_EV for a in (energies, logged, hlgaps)]
    return energies, (logged, hlgaps, mo_energy, mo_coeff, setup.coords, setup.weights)


def grad(mol, coords, weight, mo_coeff, mo_energy):
    """Nuclear gradient [Ha/Bohr], (natm, 3), of a converged SCF from its orbitals (mo_coeff,
    column k = orbital k, ascending mo_energy) on its grid (coords, weight): drop-in for
    nanoDFT.grad (nanoDFT.py:440-477; grad_elec + grad_nuc, no grid response).  Every term is
    evaluated on the B200 (b2_grad)."""
    import torch
    from .engine import NMO, Plan, _require_cuda, nuclear_gradient
    _require_cuda()
    N = mol.nao
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64).reshape(-1)).to(dev)
    plan = Plan([mol])
    try:
        plan.set_grid([len(weight)])
        eps = torch.zeros(NMO, dtype=torch.float64, device=dev)
        eps[:N] = t(np.asarray(mo_energy)[:N])
        g = nuclear_gradient(plan, t(np.asarray(mo_coeff)[:N, :N]), eps, t(coords), t(weight))
        return g.cpu().numpy().reshape(mol.natm, 3)
    finally:
        plan.close()


def main(argv=None):
    """``nanoDFT --mol_str ...`` CLI (nanoDFT.py:620-643), B200 backend, no PySCF comparison."""
    import argparse
    ap = argparse.ArgumentParser(description="nanoDFT on B200")
    ap.add_argument("--its", type=int, default=20)
    ap.add_argument("--mol_str", default="benzene")
    ap.add_argument("--float32", action="store_true")
    ap.add_argument("--basis", default="sto-3g")
    ap.add_argument("--level", type=int, default=0)
    ap.add_argument("--diis", type=lambda s: s.lower() != "false", default=True)
    a = ap.parse_args(argv)
    opts, mol_str = nanoDFT_options(its=a.its, mol_str=a.mol_str, float32=a.float32, basis=a.basis,
                                    level=a.level, diis=a.diis)
    mol = build_mol(mol_str, opts.basis)
    print(f"Number of Atomic Orbitals\t{mol.nao_nr():15d}")
    print(f"Number of electrons\t{mol.nelectron:15d}")
    E, (logged, hl, mo_e, mo_c, coords, w) = nanoDFT(mol, opts)
    print("energies [eV]:", E[:, 0])
    print("hlgap [eV]:", hl[-1])
    return E


if __name__ == "__main__":
    main()
