"""Seeded synthetic molecules with the shapes of the benchmark configurations.

The reference generates its datasets from GDB SMILES with RDKit conformers
(dft.py:236-691); neither GDB nor RDKit is available, so benchmark inputs are seeded
random trees: heavy atoms from {C, N, O, F} with given probabilities, single bonds of
length U[1.20, 1.54] A at tetrahedral angles with torsions U[0, 2pi), then hydrogens on
every free valence at 1.09 A.  Any pair of non-bonded atoms closer than 0.9 A causes a
resample.  The molecule is neutral and closed shell by construction.
"""
import numpy as np

VALENCE = {"C": 4, "N": 3, "O": 2, "F": 1}
TET = np.degrees(np.arccos(-1.0 / 3.0))      # 109.47 degrees


def _unit(v):
    return v / np.linalg.norm(v)


def _cross(a, b):
    """cross product of 3-vectors (the same arithmetic as np.cross, without its generality)"""
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _perp(u, rng):
    a = np.array([1.0, 0, 0]) if abs(u[0]) < 0.9 else np.array([0, 1.0, 0])
    p = _unit(_cross(u, a))
    q = _cross(u, p)
    phi = rng.uniform(0, 2 * np.pi)
    return np.cos(phi) * p + np.sin(phi) * q, -np.sin(phi) * p + np.cos(phi) * q


def free_directions(bonds, rng):
    """Unit vectors of the remaining tetrahedral positions around an atom."""
    b = [_unit(x) for x in bonds]
    if len(b) == 0:
        base = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], float) / np.sqrt(3)
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        return list(base @ q.T)
    if len(b) == 1:
        p, q = _perp(b[0], rng)
        ct, st = np.cos(np.radians(TET)), np.sin(np.radians(TET))
        out = []
        for k in range(3):
            a = 2 * np.pi * k / 3
            out.append(ct * b[0] + st * (np.cos(a) * p + np.sin(a) * q))
        return out
    if len(b) == 2:
        m = -_unit(b[0] + b[1])
        n = _unit(_cross(b[0], b[1]))
        be = np.radians(TET / 2)
        return [np.cos(be) * m + np.sin(be) * n, np.cos(be) * m - np.sin(be) * n]
    if len(b) == 3:
        return [-_unit(b[0] + b[1] + b[2])]
    return []


def random_molecule(rng, n_heavy, elements=("C", "N", "O", "F"), probs=(0.7, 0.1, 0.15, 0.05),
                    max_tries=1000):
    """Return an atom string (Angstrom) of a seeded random saturated tree molecule."""
    probs = np.asarray(probs, float)
    probs = probs / probs.sum()
    for _ in range(max_tries):
        syms = list(rng.choice(elements, size=n_heavy, p=probs))
        if n_heavy > 1 and sum(VALENCE[s] for s in syms) < 2 * (n_heavy - 1):
            continue
        if n_heavy > 1 and all(VALENCE[s] == 1 for s in syms):
            continue
        # order so that the root can take children: put a multivalent atom first
        if n_heavy > 1:
            k = next(i for i, s in enumerate(syms) if VALENCE[s] > 1)
            syms[0], syms[k] = syms[k], syms[0]
        pos = [np.zeros(3)]
        nbr = [[]]
        ok = True
        for a in range(1, n_heavy):
            cands = [p for p in range(a) if len(nbr[p]) < VALENCE[syms[p]] and
                     (VALENCE[syms[p]] - len(nbr[p]) > 1 or VALENCE[syms[a]] >= 1)]
            # keep at least one open valence in the tree while atoms remain to be placed
            if not cands:
                ok = False
                break
            p = cands[rng.integers(len(cands))]
            dirs = free_directions([pos[q] - pos[p] for q in nbr[p]], rng)
            d = dirs[rng.integers(len(dirs))]
            r = rng.uniform(1.20, 1.54)
            pos.append(pos[p] + r * d)
            nbr.append([p])
            nbr[p].append(a)
            if VALENCE[syms[a]] == 1 and a < n_heavy - 1:
                # a monovalent atom is a leaf; make sure the tree can still grow
                free = sum(VALENCE[syms[q]] - len(nbr[q]) for q in range(a + 1))
                if free == 0:
                    ok = False
                    break
        if not ok:
            continue
        H = []
        for a in range(n_heavy):
            nh = VALENCE[syms[a]] - len(nbr[a])
            if nh <= 0:
                continue
            dirs = free_directions([pos[q] - pos[a] for q in nbr[a]], rng)
            for d in dirs[:nh]:
                H.append(pos[a] + 1.09 * d)
        allpos = np.array(pos + H)
        allsym = syms + ["H"] * len(H)
        if len(allpos) > 1:
            d = np.sqrt(((allpos[:, None] - allpos[None]) ** 2).sum(-1))
            bonded = np.zeros_like(d, dtype=bool)
            for a in range(n_heavy):
                for q in nbr[a]:
                    bonded[a, q] = True
            np.fill_diagonal(d, np.inf)
            dd = np.where(bonded, np.inf, d)
            # hydrogens bonded to their heavy atom are at 1.09; exclude H-parent pairs
            hmin = np.inf
            iu = np.triu_indices(len(allpos), 1)
            ddu = dd[iu]
            mask = ddu > 1.0901 if False else np.ones_like(ddu, dtype=bool)
            hmin = ddu[mask].min() if mask.any() else np.inf
            # H-parent distances are exactly 1.09 -> allowed
            if hmin < 0.9:
                continue
        return "; ".join(f"{s} {x:.8f} {y:.8f} {z:.8f}" for s, (x, y, z) in zip(allsym, allpos))
    raise RuntimeError("could not generate a molecule")


def config2_molecule(seed=0):
    """9 heavy atoms from {C, N, O}, H to valence (nao <= 65)."""
    rng = np.random.default_rng(seed)
    return random_molecule(rng, 9, elements=("C", "N", "O"), probs=(0.7, 0.1, 0.15))


def config3_batch(n, seed=0, max_heavy=9):
    """n molecules, 1..max_heavy heavy atoms from {C, N, O, F} = 0.7/0.1/0.15/0.05."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        k = int(rng.integers(1, max_heavy + 1))
        out.append(random_molecule(rng, k))
    return out


def stream_molecule(seed, index, max_heavy=9):
    """Molecule ``index`` of the seeded molecule stream (1..max_heavy heavy atoms, config-3
    element probabilities); seeded per index, so any chunking gives the same stream."""
    rng = np.random.default_rng([seed, index])
    k = int(rng.integers(1, max_heavy + 1))
    return random_molecule(rng, k)


def stream_chunk(args):
    """(index, atom string, Mole) for molecules [start, start + n) of the stream, less the indices
    in an optional fifth element (molecules already written); run in worker processes (this
    module imports numpy only)"""
    from .mole import Mole
    seed, start, n, max_heavy = args[:4]
    skip = set(args[4]) if len(args) > 4 else ()
    out = []
    for i in range(start, start + n):
        if i in skip:
            continue
        s = stream_molecule(seed, i, max_heavy)
        out.append((i, s, Mole(s)))
    return out
