"""Nuclear-gradient oracle (test infrastructure: tests use it as the checker; the product never
calls it).

The reference's RKS gradient is ``grad_elec + grad_nuc`` (nanoDFT.py:403-477): derivative
integrals (int2e_ip1, int1e_ipovlp / ipkin / ipnuc / iprinv) contracted with the final density
dm0 = 2 C_occ C_occ^T and the energy-weighted density dme0 = 2 C_occ eps_occ C_occ^T, with the XC
part taken at fixed grid points and weights (no grid-response terms).  Those terms are exactly
the derivative, at fixed dm0 and a fixed grid, of

    E[dm0](R) = <dm0, T + V_nuc> + 1/2 <dm0, J[dm0]> - hyb/4 <dm0, K[dm0]> + E_xc[rho] + E_nuc

(atom A's basis functions and nucleus move with R_A; the grid does not), minus <dme0, dS/dR_A>
(the orthonormality constraint).  This oracle evaluates that derivative by central differences
of the energy expression with this repository's FP64 oracle pieces: the s8 ERI restatement
(``oracle.eri``), numpy AO values and B3LYP (``oracle.rks``) and the host 1e integrals.
Truncation error ~h^2 (h = 1e-4 Bohr: ~1e-8 Ha/Bohr).
"""
import numpy as np

from . import eri as oeri
from . import rks


def _displaced(mol, atom, axis, h):
    """the molecule with atom ``atom`` moved by h along ``axis`` (Bohr)"""
    from b200dft.mole import Mole
    xyz = mol.coords.copy()
    xyz[atom, axis] += h
    s = "; ".join(f"{sym} {x:.17g} {y:.17g} {z:.17g}" for sym, (x, y, z) in zip(mol.symbols, xyz))
    return Mole(s, basis=mol.basis, unit="Bohr", charge=mol.charge)


def energy_fixed_density(mol, D, coords, w):
    """E[D] at the molecule's geometry with density D and the grid (coords, w) held fixed;
    also returns S"""
    from b200dft.int1e import int1e
    S, T, V = int1e(mol)
    N = mol.nao
    E4 = oeri.unpack_s8(oeri.eri_s8(mol), N)
    _, J, K = rks.get_JK(D, E4)
    ao = rks.ao_values(mol, coords)
    E_xc, _, _ = rks.exchange_correlation(D, ao, w)
    E = (float((D * (T + V)).sum()) + 0.5 * float((D * J).sum()) - rks.HYB / 4 * float((D * K).sum())
         + E_xc + mol.energy_nuc())
    return E, S


def gradient(mol, mo_coeff, mo_energy, coords, w, h=1e-4):
    """(natm, 3) gradient [Ha/Bohr] of the reference's formula (nanoDFT.py:403-477) for the
    orbitals (mo_coeff, columns, ascending mo_energy) of a converged SCF on the grid (coords, w)"""
    nocc = mol.nelectron // 2
    C = mo_coeff[:, :nocc]
    dm0 = 2 * C @ C.T
    dme0 = 2 * (C * mo_energy[:nocc]) @ C.T
    g = np.zeros((mol.natm, 3))
    for a in range(mol.natm):
        for x in range(3):
            Ep, Sp = energy_fixed_density(_displaced(mol, a, x, h), dm0, coords, w)
            Em, Sm = energy_fixed_density(_displaced(mol, a, x, -h), dm0, coords, w)
            g[a, x] = (Ep - Em) / (2 * h) - float((dme0 * (Sp - Sm)).sum()) / (2 * h)
    return g
