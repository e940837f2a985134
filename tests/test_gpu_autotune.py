"""The XC tile autotuner on the B200: every bucket of a small uneven batch gets a candidate, and
the tuned launches give the same V_xc / E_xc as the default split."""
import numpy as np
import pytest
import torch

from b200dft import autotune
from b200dft.engine import RKSEngine
from b200dft.mole import Mole
from b200dft.molgen import config3_batch

pytestmark = pytest.mark.gpu


def test_autotune_xc_tiles(cuda):
    mols = [Mole(s) for s in config3_batch(96, seed=3)]
    eng = RKSEngine(mols, precision="mixed", guess="minao", tuned=False)
    eng.prepare()
    eng.D.copy_(eng.D0)
    eng.xc()
    torch.cuda.synchronize()
    e0, v0 = eng.exc.cpu().numpy().copy(), eng.Vxc.cpu().numpy().copy()
    choice, times = autotune.tune_xc_tiles(eng, candidates=(1, 4, 16), reps=2)
    buckets = {autotune.bucket_of(n) for n in eng.plan.nao}
    assert set(choice) == buckets and all(c in (1, 4, 16) for c in choice.values())
    assert all(len(times[b]) == 3 for b in buckets)
    eng.xc()
    torch.cuda.synchronize()
    np.testing.assert_allclose(eng.exc.cpu().numpy(), e0, rtol=1e-6)
    np.testing.assert_allclose(eng.Vxc.cpu().numpy(), v0, atol=1e-5 * np.abs(v0).max())
    eng.close()
