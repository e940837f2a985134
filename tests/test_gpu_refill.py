"""Slot refill (b200dft.refill.run_refill) on the B200: every molecule of a stream converges to
the same energy as in whole batches (run_batches), with molecules carried across plans mid-SCF."""
import numpy as np
import pytest

from b200dft.engine import run_batches
from b200dft.mole import Mole
from b200dft.molgen import config3_batch
from b200dft.refill import run_refill

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("guess,graph", [("minao", False), ("learned", False), ("learned", True)])
def test_refill_matches_whole_batches(cuda, guess, graph):
    # eager SCF steps (the default) and one captured graph per refill plan give the same results
    mols = [Mole(s) for s in config3_batch(320, seed=5)]
    ref = np.zeros(len(mols))
    rconv = np.zeros(len(mols), bool)
    k = 0
    for ms, out in run_batches([mols[i:i + 160] for i in range(0, len(mols), 160)], guess=guess):
        ref[k:k + len(ms)] = out["energy"]
        rconv[k:k + len(ms)] = out["converged"]
        k += len(ms)
    got = np.full(len(mols), np.nan)
    conv = np.zeros(len(mols), bool)
    refills = 0
    for ids, ms, out in run_refill(iter(mols), slots=96, refill_at=0.5, guess=guess, graph=graph):
        got[ids] = out["energy"]
        conv[ids] = out["converged"]
        assert all(mols[i] is m for i, m in zip(ids, ms))
        assert np.all(np.isfinite(out["last5"][out["converged"]][:, -1]))
        refills += 1
    assert refills >= 3                          # slots were refilled several times
    assert not np.isnan(got).any()
    assert conv.sum() >= rconv.sum() - 1
    both = conv & rconv
    assert np.abs(got[both] - ref[both]).max() < 1e-5
