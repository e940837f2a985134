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
