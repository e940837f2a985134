"""bench.py host logic that runs without a GPU."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402
from b200dft.mole import Mole, methane  # noqa: E402


def test_quartet_counts_match_enumeration():
    mols = [Mole(methane()), Mole("N 0 0 0; C 0 0 2.6; O 2.1 0 3.9; H 0 1.9 -0.8", unit="Bohr")]
    q, p = bench.quartet_counts(mols)
    qb = pb = 0
    for m in mols:
        npr = [int(b[2]) for b in m._bas]
        pairs = [(i, j) for i in range(len(npr)) for j in range(i + 1)]
        for a in range(len(pairs)):
            for b in range(a + 1):
                qb += 1
                (i, j), (k, l) = pairs[a], pairs[b]
                pb += npr[i] * npr[j] * npr[k] * npr[l]
    assert (q, p) == (qb, pb)
    assert bench.quartet_counts([Mole(methane())]) == (406, 406 * 81)   # 7 shells, 3 primitives each


def test_reference_arm_json_contract():
    """bench.py --impl reference (the CPU path, no GPU needed) prints one JSON line with the
    contract's keys"""
    import json
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_reference_arm_other_ranks_exit_quietly():
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=root, env=env)
    assert r.returncode == 0 and not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_parity_eri_difference_skips_padding():
    """max |dERI| of the parity leg covers each molecule's s8 entries and skips the padding to the
    next 32-entry offset (never written by the kernels)"""
    import types
    import torch
    plan = types.SimpleNamespace(eri_off=np.array([0, 32, 96]), nao=np.array([2, 3, 2], np.int32))
    # n2 = 3, 6, 3 -> n4 = 6, 21, 6 entries per molecule
    x = torch.zeros(128, dtype=torch.float32)
    y = torch.zeros(128, dtype=torch.float64)
    x[6:32] = 5.0                  # padding of molecule 0
    x[32 + 21:96] = 7.0            # padding of molecule 1
    x[96 + 6:] = 9.0               # past the last molecule
    x[40] = 0.25                   # a real difference in molecule 1
    y[100] = -0.5                  # and one in molecule 2
    assert bench._max_abs_diff_lists(x, y, plan, step=50) == 0.5
    y[100] = 0.0
    assert bench._max_abs_diff_lists(x, y, plan, step=7) == 0.25
