"""The C ABI library loads and exports every symbol declared in include/b200dft.h (CPU)."""
import ctypes
import os
import re

from conftest import ROOT
from b200dft._lib import LIB_PATH, SIGNATURES


def declared():
    src = open(os.path.join(ROOT, "include", "b200dft.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(b2_\w+)\s*\(", src, re.M)))


def test_header_declares_all_bound():
    names = declared()
    assert len(names) >= 18
    for n in SIGNATURES:
        assert n in names, n


def test_library_exports_all_declared():
    assert os.path.exists(LIB_PATH), "build with pyscf-ipu_b200/csrc/build.py"
    lib = ctypes.CDLL(LIB_PATH)              # loading needs no GPU
    for n in declared():
        assert hasattr(lib, n), n
    assert lib.b2_version() >= 100


def test_no_cpu_fallback():
    # the product entry refuses to run without a device instead of computing on the CPU
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    from b200dft.engine import RKSEngine
    from b200dft.mole import Mole, methane
    from b200dft._lib import B200DFTError
    with pytest.raises(B200DFTError):
        RKSEngine([Mole(methane())])


def test_noalloc_rejects_bad_arguments_without_a_gpu():
    # b2_int2e_sph_s8_noalloc checks its host arguments before any CUDA call: a negative or
    # out-of-range exponent / coefficient offset is B2_ERR_ARG, too many shells B2_ERR_SIZE
    import numpy as np
    from b200dft._lib import lib, ptr
    from b200dft.mole import Mole, methane
    m = Mole(methane())
    env = np.ascontiguousarray(m._env)
    out = ctypes.c_void_p(16)                 # never dereferenced: every case fails its checks first
    for slot, value in ((5, -1), (6, -3), (5, len(env))):        # PTR_EXP, PTR_COEFF
        bas = np.array(m._bas, np.int32)
        bas[0, slot] = value
        atm = np.ascontiguousarray(m._atm, np.int32)
        rc = lib().b2_int2e_sph_s8_noalloc(ptr(atm), m.natm, ptr(bas), m.nbas, ptr(env), len(env), 64,
                                           out, None)
        assert rc == -1, (slot, value, rc)
    big = Mole("; ".join(f"H {x * 1.5} 0 0" for x in range(50)))
    rc = lib().b2_int2e_sph_s8_noalloc(ptr(np.ascontiguousarray(big._atm, np.int32)), big.natm,
                                       ptr(np.ascontiguousarray(big._bas, np.int32)), big.nbas,
                                       ptr(np.ascontiguousarray(big._env)), len(big._env), 64, out, None)
    assert rc == -4
