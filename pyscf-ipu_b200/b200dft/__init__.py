"""b200dft: a B200-native restricted Kohn-Sham (B3LYP/STO-3G) SCF engine.

Drop-in for the RKS hot path of pyscf-ipu: ``density_functional_theory`` (pyscf_ipu/dft.py:197)
and ``nanoDFT`` (pyscf_ipu/nanoDFT/nanoDFT.py:259).  Host setup (molecule, basis, grid,
one-electron matrices, guess) runs in Python/numpy; ERIs, J/K, the XC grid path and the
SCF loop run in hand-written sm_100a CUDA kernels behind a C ABI (libb200dft.so).
"""
from .constants import HARTREE_TO_EV, HYB_B3LYP, EPSILON_B3LYP
from .mole import Mole, build_mol, methane

__all__ = ["Mole", "build_mol", "methane", "HARTREE_TO_EV", "HYB_B3LYP", "EPSILON_B3LYP"]
