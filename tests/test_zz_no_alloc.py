"""The allocation-free ERI entry point (b2_int2e_sph_s8_noalloc) against b2_int2e_sph_s8.

Callers that must not call cudaMalloc (device memory owned by another allocator or a
fixed-budget pool, loops where an allocation could block or synchronise the device) use the
no-alloc entry; it must give the same s8 list as the allocating entry, and keep doing so on
consecutive calls that reuse its static device array.
Collected last so that a failure here does not hide the rest of the GPU suite.
"""
import numpy as np
import pytest
import torch

from b200dft.mole import Mole, methane
from b200dft.molgen import random_molecule
from b200dft._lib import lib, check, ptr, stream_handle

pytestmark = pytest.mark.gpu


def _n_s8(nao):
    n2 = nao * (nao + 1) // 2
    return n2 * (n2 + 1) // 2


def _call(name, m, prec):
    assert torch.cuda.is_available()
    dt = torch.float64 if prec == 64 else torch.float32
    out = torch.full((_n_s8(m.nao),), float("nan"), dtype=dt, device="cuda")
    atm = np.ascontiguousarray(m._atm, np.int32)
    bas = np.ascontiguousarray(m._bas, np.int32)
    env = np.ascontiguousarray(m._env)
    check(getattr(lib(), name)(ptr(atm), m.natm, ptr(bas), m.nbas, ptr(env), len(env), prec, ptr(out),
                               stream_handle()), name)
    torch.cuda.synchronize()
    return out.double().cpu().numpy()


@pytest.mark.parametrize("prec", [64, 32])
def test_noalloc_matches_allocating_entry(prec):
    rng = np.random.default_rng(17)
    mols = [Mole(methane()), Mole(random_molecule(rng, 6))]
    tol = 1e-10 if prec == 64 else 5e-6
    for m in mols:                                     # two calls in a row through the static array
        ref = _call("b2_int2e_sph_s8", m, prec)
        got = _call("b2_int2e_sph_s8_noalloc", m, prec)
        assert not np.isnan(got).any()
        np.testing.assert_allclose(got, ref, atol=tol, rtol=0)


def test_noalloc_rejects_oversize():
    # 49 shells exceed the static array's limit: clear error, nothing launched
    s = "; ".join(f"H {x * 1.5} 0 0" for x in range(50))
    m = Mole(s)
    atm = np.ascontiguousarray(m._atm, np.int32)
    bas = np.ascontiguousarray(m._bas, np.int32)
    env = np.ascontiguousarray(m._env)
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib().b2_int2e_sph_s8_noalloc(ptr(atm), m.natm, ptr(bas), m.nbas, ptr(env), len(env), 64,
                                       ptr(out), stream_handle())
    assert rc == -4
