"""STO-3G basis data and libcint-convention normalisation.

Exponents and contraction coefficients are the published STO-3G values
(Hehre, Stewart, Pople, J. Chem. Phys. 51, 2657 (1969); Hehre, Ditchfield,
Stewart, Pople, J. Chem. Phys. 52, 2769 (1970)).  The reference takes them from
PySCF's basis library (``mol.build(basis="sto-3g")``, pyscf_utils/build_mol.py:5,
nanoDFT.py:543-546).  As in PySCF, the 2sp shell of a heavy atom is split into
an s shell and a p shell with shared exponents, and shells are ordered by
angular momentum inside an atom, so a heavy atom carries AOs
[1s, 2s, 2px, 2py, 2pz] and hydrogen [1s].

Normalisation follows libcint: ``env`` holds coefficients c_i * N(l, a_i)
rescaled so the contracted radial function R(r) = sum_i c'_i r^l exp(-a_i r^2)
has int R^2 r^2 dr = 1; the angular factor 1/sqrt(4 pi) (s) or sqrt(3/(4 pi)) (p)
is applied by the integral code (cpu_int2e_sph.cpp, CINTcommon_fac_sp).
"""
import functools
import math
import numpy as np

_S1 = (0.15432897, 0.53532814, 0.44463454)
_S2 = (-0.09996723, 0.39951283, 0.70011547)
_P2 = (0.15591627, 0.60768372, 0.39195739)

# element -> list of (l, exponents, coefficients)
STO3G = {
    "H": [(0, (3.42525091, 0.62391373, 0.16885540), _S1)],
    "C": [(0, (71.6168370, 13.0450960, 3.5305122), _S1),
          (0, (2.9412494, 0.6834831, 0.2222899), _S2),
          (1, (2.9412494, 0.6834831, 0.2222899), _P2)],
    "N": [(0, (99.1061690, 18.0523120, 4.8856602), _S1),
          (0, (3.7804559, 0.8784966, 0.2857144), _S2),
          (1, (3.7804559, 0.8784966, 0.2857144), _P2)],
    "O": [(0, (130.7093200, 23.8088610, 6.4436083), _S1),
          (0, (5.0331513, 1.1695961, 0.3803890), _S2),
          (1, (5.0331513, 1.1695961, 0.3803890), _P2)],
    "F": [(0, (166.6791300, 30.3608120, 8.2168207), _S1),
          (0, (6.4648032, 1.5022812, 0.4885885), _S2),
          (1, (6.4648032, 1.5022812, 0.4885885), _P2)],
}

BASIS_SETS = {"sto-3g": STO3G, "sto3g": STO3G}


def gaussian_int(n, a):
    """int_0^inf r^n exp(-a r^2) dr."""
    n1 = (n + 1) * 0.5
    return math.gamma(n1) / (2.0 * a ** n1)


def gto_norm(l, a):
    """Radial normalisation of r^l exp(-a r^2) over r^2 dr."""
    return 1.0 / math.sqrt(gaussian_int(2 * l + 2, 2.0 * a))


def normalized_coefficients(l, exps, coefs):
    """libcint-convention contracted coefficients (radial part normalised to 1); cached per
    shell (a basis has few distinct shells, every molecule reuses them)"""
    return np.array(_normalized_coefficients(int(l), tuple(float(a) for a in exps),
                                             tuple(float(c) for c in coefs)))


@functools.lru_cache(maxsize=None)
def _normalized_coefficients(l, exps, coefs):
    exps = np.asarray(exps, dtype=np.float64)
    cs = np.asarray(coefs, dtype=np.float64) * np.array([gto_norm(l, a) for a in exps])
    ee = exps[:, None] + exps[None, :]
    ovl = np.vectorize(lambda a: gaussian_int(2 * l + 2, a))(ee)
    s = cs @ ovl @ cs
    return tuple((cs / math.sqrt(s)).tolist())


def get_basis(name):
    key = name.lower().replace("_", "-")
    if key not in BASIS_SETS:
        raise ValueError(f"basis '{name}' is not supported (only STO-3G)")
    return BASIS_SETS[key]
