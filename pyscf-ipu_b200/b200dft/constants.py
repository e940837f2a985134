"""Physical constants and libcint slot layout used across the package.

The slot constants follow the libcint ``atm``/``bas``/``env`` layout that the
reference packs for its ERI kernels (pyscf_ipu/electron_repulsion/cpu_int2e_sph.cpp:47-88,
pyscf_ipu/electron_repulsion/direct.py:710-739).
"""
import math

BOHR_ANGSTROM = 0.52917721092          # 1 Bohr in Angstrom
ANGSTROM_TO_BOHR = 1.0 / BOHR_ANGSTROM
HARTREE_TO_EV = 27.2114079527          # nanoDFT.py:16
HYB_B3LYP = 0.2                        # nanoDFT.py:18
EPSILON_B3LYP = 1e-20                  # nanoDFT.py:17
CLIP_RHO_MIN = 1e-9                    # b3lyp.py:10
CLIP_RHO_MAX = 1e12                    # b3lyp.py:11

# libcint env / atm / bas slots (cpu_int2e_sph.cpp:47-88)
PTR_EXPCUTOFF = 0
PTR_ENV_START = 20
CHARGE_OF, PTR_COORD, NUC_MOD_OF, PTR_ZETA = 0, 1, 2, 3
ATM_SLOTS = 6
ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, KAPPA_OF, PTR_EXP, PTR_COEFF = 0, 1, 2, 3, 4, 5, 6
BAS_SLOTS = 8

# real-solid-harmonic angular normalisation applied by libcint on top of the
# radial normalisation stored in env (CINTcommon_fac_sp)
COMMON_FAC_SP = {0: 0.5 / math.sqrt(math.pi), 1: math.sqrt(3.0 / (4.0 * math.pi))}

ELEMENTS = {"H": 1, "He": 2, "C": 6, "N": 7, "O": 8, "F": 9}
SYMBOLS = {v: k for k, v in ELEMENTS.items()}
