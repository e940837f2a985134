"""Tile autotuner for the batched engine's kernels (project-written; no counterpart in the
reference, whose IPU path fixes its tile/thread split by hand, electron_repulsion/direct.py:
584-707 and nanoDFT/sparse_symmetric_ERI.py:36-64).

Knob: grid tiles (128 points) per work item of the per-bucket tensor-core XC kernel, chosen
separately for each orbital bucket (nao <= 16, 32, 48, 64, more).  Few tiles per item balance
the work queue; many amortise the per-item load of D and the flush of V.  ``tune_xc_tiles``
times ``b2_xc_direct`` on the molecules of one bucket at a time (the others inactive) for every
candidate, with CUDA events, and keeps the fastest.  The choices are recorded per device in
``tuned.json`` beside this file (``save``), and ``RKSEngine`` applies the recorded table of its
device to every new plan (``apply``).
"""
import json
import os

import numpy as np

from ._lib import lib, check, ptr

NBKT = 5
CANDIDATES = (1, 2, 4, 8, 16, 32, 64)
TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")


def bucket_of(nao):
    """orbital bucket of a molecule (the kernels' grouping: nao <= 16, 32, 48, 64, more)"""
    return min(NBKT - 1, (int(nao) - 1) // 16)


def pick(times):
    """times: {bucket: {candidate: ms}} -> {bucket: fastest candidate} (ties: fewer tiles)"""
    return {b: min(sorted(t), key=lambda c: (t[c], c)) for b, t in times.items() if t}


def tiles_array(choice):
    """int32[5] for b2_plan_set_xc_bucket_tiles (0 = the plan-wide default)"""
    a = np.zeros(NBKT, np.int32)
    for b, c in choice.items():
        a[int(b)] = int(c)
    return a


def set_bucket_tiles(plan, choice):
    check(lib().b2_plan_set_xc_bucket_tiles(plan.h, ptr(tiles_array(choice))), "b2_plan_set_xc_bucket_tiles")
    plan.epoch += 1


def tune_xc_tiles(eng, candidates=CANDIDATES, reps=3):
    """Time the XC entry of ``eng`` (setup and density in place) per bucket and candidate;
    returns (choice {bucket: tiles}, times {bucket: {tiles: ms}}).  Leaves the choice applied."""
    import torch
    P = eng.plan
    bk = np.array([bucket_of(n) for n in P.nao])
    times = {}
    for b in range(NBKT):
        sel = bk == b
        if not sel.any():
            continue
        act = torch.from_numpy(sel.astype(np.int32)).to(eng.device)
        times[b] = {}
        for c in candidates:
            set_bucket_tiles(P, {b: c})
            eng.xc(active=act)                       # warm-up (first use of the items)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps)]
            ms = []
            for r in range(reps):
                ev[2 * r].record()
                eng.xc(active=act)
                ev[2 * r + 1].record()
            torch.cuda.synchronize()
            ms = [ev[2 * r].elapsed_time(ev[2 * r + 1]) for r in range(reps)]
            times[b][c] = float(np.median(ms))
    choice = pick(times)
    set_bucket_tiles(P, choice)
    return choice, times


def device_key():
    import torch
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


_CACHE = {}


def load(path=TABLE, cached=False):
    if cached and path in _CACHE:
        return _CACHE[path]
    d = {}
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
    _CACHE[path] = d
    return d


def save(choice, times, key, path=TABLE, workload=""):
    d = load(path)
    d[key] = {"xc_tiles": {str(b): int(c) for b, c in choice.items()},
              "xc_ms": {str(b): {str(c): round(v, 4) for c, v in t.items()} for b, t in times.items()},
              "workload": workload}
    with open(path, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


def apply(plan, key=None, path=TABLE):
    """apply the recorded XC tile choice of this device (if any) to ``plan``; returns it"""
    t = load(path, cached=True).get(key or device_key())
    if not t:
        return None
    choice = {int(b): int(c) for b, c in t.get("xc_tiles", {}).items()}
    if choice:
        set_bucket_tiles(plan, choice)
    return choice


def main(argv=None):
    """python -m b200dft.autotune [--nmol N]: tune on a seeded batch of the batched workload and
    record the choice for this device"""
    import argparse
    from .engine import RKSEngine
    from .mole import Mole
    from .molgen import config3_batch
    ap = argparse.ArgumentParser()
    ap.add_argument("--nmol", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--no-save", action="store_true")
    ap.add_argument("--out", default=TABLE, help="table file to record the choice in")
    a = ap.parse_args(argv)
    mols = [Mole(s) for s in config3_batch(a.nmol, seed=a.seed)]
    eng = RKSEngine(mols, precision="mixed", guess="minao", tuned=False)
    try:
        eng.prepare()
        eng.D.copy_(eng.D0)
        choice, times = tune_xc_tiles(eng)
    finally:
        eng.close()
    print(json.dumps({"choice": choice, "times_ms": times}))
    if not a.no_save:
        save(choice, times, device_key(), path=a.out,
             workload=f"{a.nmol} molecules, config-3 distribution, seed {a.seed}")


if __name__ == "__main__":
    main()
