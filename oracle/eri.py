"""ctypes access to the ERI oracle libraries (test infrastructure).

``eri_s8`` runs this project's FP64 C restatement (eri_oracle.c); ``ref_eri_s8`` runs the
reference's own FP64 ``int2e_sph`` (cpu_int2e_sph.cpp:7706) through ref_s8_driver.c.  Both
return the s8 unique-ERI list of ``mol.intor('int2e_sph', aosym='s8')`` (nanoDFT.py:285).
"""
import ctypes
import os
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle_eri.so")
_REF = os.path.join(HERE, "_ref", "libref_s8.so")
_lib = None
_ref = None


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.oracle_eri_s8.restype = ctypes.c_int
    return _lib


def ref_available():
    return os.path.exists(_REF)


def reflib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(_REF + " (build with oracle/build_ref.py where the reference is present)")
        _ref = ctypes.CDLL(_REF)
    return _ref


def n_s8(nao):
    n2 = nao * (nao + 1) // 2
    return n2 * (n2 + 1) // 2


def _arrays(mol):
    atm = np.ascontiguousarray(mol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(mol._bas, dtype=np.int32)
    env = np.ascontiguousarray(mol._env, dtype=np.float64)
    ao_loc = np.ascontiguousarray(mol.ao_loc, dtype=np.int32)
    return atm, bas, env, ao_loc


def eri_s8(mol):
    atm, bas, env, ao_loc = _arrays(mol)
    out = np.zeros(n_s8(mol.nao), dtype=np.float64)
    lib().oracle_eri_s8(_p(out, ctypes.c_double), _p(ao_loc, ctypes.c_int), _p(atm, ctypes.c_int),
                        ctypes.c_int(mol.natm), _p(bas, ctypes.c_int), ctypes.c_int(mol.nbas),
                        _p(env, ctypes.c_double))
    return out


def ref_eri_s8(mol):
    atm, bas, env, ao_loc = _arrays(mol)
    out = np.zeros(n_s8(mol.nao), dtype=np.float64)
    reflib().ref_eri_s8(_p(out, ctypes.c_double), _p(ao_loc, ctypes.c_int), _p(atm, ctypes.c_int),
                        ctypes.c_int(mol.natm), _p(bas, ctypes.c_int), ctypes.c_int(mol.nbas),
                        _p(env, ctypes.c_double), ctypes.c_int(len(env)))
    return out


def ref_int2e_block(mol, shls):
    atm, bas, env, _ = _arrays(mol)
    out = np.zeros(256, dtype=np.float64)
    sh = np.asarray(shls, dtype=np.int32)
    reflib().ref_int2e_block(_p(out, ctypes.c_double), ctypes.c_int(256), _p(sh, ctypes.c_int),
                             _p(atm, ctypes.c_int), ctypes.c_int(mol.natm), _p(bas, ctypes.c_int),
                             ctypes.c_int(mol.nbas), _p(env, ctypes.c_double), ctypes.c_int(len(env)))
    return out


def boys(mmax, t):
    f = np.zeros(mmax + 1)
    lib().oracle_boys(ctypes.c_int(mmax), ctypes.c_double(t), _p(f, ctypes.c_double))
    return f


def unpack_s8(s8, nao):
    """s8 list -> dense (nao,nao,nao,nao) tensor (all 8 permutations)."""
    i, j = np.tril_indices(nao)
    n2 = len(i)
    M = np.zeros((n2, n2))
    r, c = np.tril_indices(n2)
    M[r, c] = s8
    M[c, r] = s8
    E = np.zeros((nao, nao, nao, nao))
    A = np.zeros((nao, nao, n2))
    A[i, j, np.arange(n2)] = 1
    A[j, i, np.arange(n2)] = 1
    E = np.einsum("abp,pq,cdq->abcd", A, M, A, optimize=True)
    return E
