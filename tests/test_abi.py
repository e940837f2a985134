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
