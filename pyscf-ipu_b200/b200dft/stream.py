"""Streaming dataset generation: a molecule stream through the batched B200 SCF into rows.

Restates the reference's generation driver (dft.py:236-691): molecules are taken from a
stream, each gets a B3LYP/STO-3G SCF, and one row per molecule is appended to the output
with the energy, HOMO, LUMO and HOMO-LUMO gap in eV, the standard deviation of the energies of
the last five iterations (the reference's convergence column, dft.py:632) and N = nao.  Two
output schemas:

* ``parquet``: the QM1B schema (qm1b/README.md:5-19): smile, atoms, z, energy, homo, lumo, N,
  std, y (= gap), pos (Bohr, flattened), plus ``iterations`` and ``converged``;
* ``csv``: gzip CSV with the reference's row dictionary (dft.py:629-645) where the data exist
  here: smile, atoms, atom_positions, energies (last five, eV), std, homo, lumo, hlgap, N, basis.

Molecules come from the seeded synthetic generator (``molgen.random_molecule``, the stand-in for
the GDB-11 SMILES + RDKit conformers the reference reads, which are not available); the
``smile`` column therefore holds an identifier ``gen:<seed>:<index>:<formula>``.

Pipelining (the reference overlaps host preparation with device compute the same way): a
``spawn`` process pool generates and parses molecules in chunks of one batch; a host thread
keeps the next batch ready while the GPU runs the current one (the workers also make each
molecule's static row columns); ``engine.run_batches`` runs the batches, building each next plan
on its worker thread once the current batch's ERI work is queued; a writer thread converts and
appends finished batches (result columns by numpy).  Each batch is one ``RKSEngine`` run to
convergence: molecules retire individually as they converge (their kernels skip them, and the
J/K and XC launches are compacted to the stragglers), so a batch ends when its slowest molecule
converges.
"""
import argparse
import collections
import json
import multiprocessing as mp
import os
import queue
import threading
import time
from collections import Counter

import numpy as np
import torch

from .constants import HARTREE_TO_EV
from .engine import run_batches
from .mole import pack_moles, unpack_moles
from .molgen import stream_chunk

QM1B_COLUMNS = ("smile", "atoms", "z", "energy", "homo", "lumo", "N", "std", "y", "pos")


def _formula(symbols):
    c = Counter(symbols)
    return "".join(f"{e}{c[e] if c[e] > 1 else ''}" for e in sorted(c, key=lambda e: (e != "C", e != "H", e)))


def static_columns(idx, m, seed):
    """the columns of one molecule that do not depend on its SCF (computed where the molecule is
    generated, in the worker processes)"""
    return {"smile": f"gen:{seed}:{idx}:{_formula(m.symbols)}", "atoms": "".join(m.symbols),
            "z": [int(z) for z in m.charges], "pos": [float(x) for x in m.coords.reshape(-1)]}


def _low_priority():
    """worker initialiser: generation yields the cores to the process that drives the GPU"""
    try:
        os.nice(10)
    except OSError:
        pass


def done_indices(path, fmt, seed):
    """indices of the molecules of stream ``seed`` whose rows ``path`` already holds (from the
    rows' identifiers gen:<seed>:<index>:<formula>); the reference's generation loop skips the
    molecules found in its output folder the same way (dft.py:247-283, option -resume)"""
    import os
    if not path or not os.path.exists(path):
        return set()
    if fmt == "parquet":
        import pyarrow.parquet as pq
        smiles = pq.read_table(path, columns=["smile"]).column("smile").to_pylist()
    else:
        import pandas as pd
        smiles = pd.read_csv(path, compression="gzip", usecols=["smile"])["smile"].tolist()
    out = set()
    for s in smiles:
        p = str(s).split(":")
        if len(p) >= 3 and p[0] == "gen" and p[1] == str(seed):
            out.add(int(p[2]))
    return out


def prepare_chunk(args):
    """worker: molecules of one chunk of the stream with their static columns; the molecules
    travel packed (``unpack_chunk`` on the receiving side)"""
    items = stream_chunk(args)
    return [(i, s, static_columns(i, m, args[0])) for i, s, m in items], pack_moles([m for _, _, m in items])


def unpack_chunk(chunk):
    """(index, atom string, Mole, static columns) per molecule of a chunk from ``prepare_chunk``"""
    meta, packed = chunk
    return [(i, s, m, st) for (i, s, st), m in zip(meta, unpack_moles(packed))]


def batch_rows(items, res, seed):
    """rows (dict of columns) of one finished batch; the per-molecule static columns come with
    the items when the workers made them, else they are made here"""
    n = len(items)
    h = lambda x: x.cpu().numpy() if torch.is_tensor(x) else np.asarray(x)
    E = h(res["energy"]) * HARTREE_TO_EV
    mo = h(res["mo_energy"]).reshape(n, -1)
    last5 = h(res["last5"]) * HARTREE_TO_EV
    its = h(res["iterations"])
    conv = h(res["converged"])
    mols = [it[2] for it in items]
    nocc = np.array([m.nelectron // 2 for m in mols], np.int64)
    nao = np.array([m.nao for m in mols], np.int64)
    r = np.arange(n)
    homo = mo[r, nocc - 1] * HARTREE_TO_EV
    lumo = np.where(nocc < nao, mo[r, np.minimum(nocc, mo.shape[1] - 1)] * HARTREE_TO_EV, np.nan)
    fin = np.isfinite(last5)
    cnt = fin.sum(1)
    l5 = np.where(fin, last5, 0.0)
    mean = l5.sum(1) / np.maximum(cnt, 1)
    std = np.sqrt((np.where(fin, last5 - mean[:, None], 0.0) ** 2).sum(1) / np.maximum(cnt, 1))
    std = np.where(cnt > 0, std, np.nan)
    stat = [it[3] if len(it) > 3 else static_columns(it[0], it[2], seed) for it in items]
    cols = {k: [st[k] for st in stat] for k in ("smile", "atoms", "z", "pos")}
    cols.update({"energy": E.tolist(), "homo": homo.tolist(), "lumo": lumo.tolist(), "N": nao.tolist(),
                 "std": std.tolist(), "y": np.abs(lumo - homo).tolist(), "iterations": its.astype(int).tolist(),
                 "converged": conv.astype(bool).tolist(),
                 "last5": [row[f].tolist() for row, f in zip(last5, fin)]})
    if "gradient" in res:
        # nuclear gradient dE/dR (Ha/Bohr) of each molecule, flattened like pos
        g = h(res["gradient"]).reshape(-1, 3)
        a0 = np.concatenate([[0], np.cumsum([m.natm for m in mols])])
        cols["gradient"] = [g[a0[k]:a0[k + 1]].reshape(-1).tolist() for k in range(n)]
    return cols


class RowWriter:
    """Appends batches of rows to a Parquet file (QM1B schema) or a gzip CSV (reference schema)."""

    def __init__(self, path, fmt="parquet", basis="sto-3g", append=False):
        import os
        self.path, self.fmt, self.basis = path, fmt, basis
        self._pq = None
        self._first = True
        self._prior = None                    # rows already in a Parquet file being appended to
        if append and path and os.path.exists(path):
            if fmt == "parquet":
                import pyarrow.parquet as pq
                self._prior = pq.read_table(path)
            else:
                self._first = False           # gzip CSV: append members, no second header

    def write(self, cols):
        if self.path is None:
            return
        if self.fmt == "parquet":
            import pyarrow as pa
            import pyarrow.parquet as pq
            keep = QM1B_COLUMNS + ("iterations", "converged") + (("gradient",) if "gradient" in cols else ())
            t = pa.table({k: cols[k] for k in keep})
            if self._pq is None:
                if self._prior is not None:
                    # a Parquet file cannot be appended in place: rewrite its rows first
                    if self._prior.schema.names != t.schema.names:
                        raise ValueError(f"{self.path} has columns {self._prior.schema.names}, new rows {t.schema.names}")
                    t = pa.concat_tables([self._prior.cast(t.schema), t])
                    self._prior = None
                self._pq = pq.ParquetWriter(self.path, t.schema)
            self._pq.write_table(t)
        else:
            import pandas as pd
            df = pd.DataFrame({
                "smile": cols["smile"], "atoms": cols["atoms"], "atom_positions": cols["pos"],
                "energies": cols["last5"], "std": cols["std"], "homo": cols["homo"],
                "lumo": cols["lumo"], "hlgap": cols["y"], "N": cols["N"],
                "basis": [self.basis] * len(cols["N"])})
            if "gradient" in cols:
                df["gradient"] = cols["gradient"]
            df.to_csv(self.path, mode="a", header=self._first, compression="gzip")
            self._first = False

    def close(self):
        self._prior = None                           # nothing new written: the file is untouched
        if self._pq is not None:
            self._pq.close()
            self._pq = None


def run_stream(n_total, batch=4096, seed=0, level=0, precision="mixed", guess="learned", out=None,
               fmt="parquet", workers=None, max_heavy=9, net=None, e_tol=1e-6, diis_tol=1e-4,
               rank=0, world=1, gradient=False, resume=False, refill=False):
    """Generate ``n_total`` molecules and write one row each; returns throughput and iteration
    statistics (the streaming configuration: molecules/s, p50/p99 iterations).  With
    ``world`` > 1 this process handles the stream chunks of ``rank`` (round robin) only.  With
    ``gradient`` each row also carries the molecule's nuclear gradient (force labels, dE/dR in
    Ha/Bohr, flattened like ``pos``; nanoDFT.py:440-477 on the SCF's final orbitals).  With
    ``resume`` the molecules whose rows ``out`` already holds are not generated again and the new
    rows are appended (dft.py:247-283).  With ``refill`` the batch's slots are refilled from the
    stream as molecules converge (b200dft.refill.run_refill) instead of running whole batches."""
    if refill and gradient:
        raise ValueError("force labels are computed per whole batch: use refill=False with gradient")
    if guess == "learned" and net is None:
        from .train_guess import load
        net = load()
    workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
    from .shard import shard_indices
    chunks = [(seed, s, min(batch, n_total - s), max_heavy) for s in shard_indices(n_total, batch, rank, world)]
    skipped = 0
    if resume:
        done_idx = np.array(sorted(done_indices(out, fmt, seed)), np.int64)
        kept = []
        for c in chunks:
            lo, hi = np.searchsorted(done_idx, [c[1], c[1] + c[2]])
            skipped += int(hi - lo)
            if hi - lo < c[2]:                    # chunks fully written are not generated again
                kept.append(c + (tuple(int(i) for i in done_idx[lo:hi]),))
        chunks = kept
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(workers, initializer=_low_priority)
    ready = queue.Queue(maxsize=2)        # generated batches waiting for the GPU
    done = queue.Queue(maxsize=4)         # finished batches waiting for the writer
    writer = RowWriter(out, fmt, append=resume)
    stats = {"iterations": [], "converged": 0, "batches": 0, "gpu_s": 0.0}
    err = []

    def submit(c):
        # one batch split over every worker (with the indices each piece skips, if resuming)
        seed_, start, n, mh = c[:4]
        skip = c[4] if len(c) > 4 else ()
        step = max(1, -(-n // workers))
        return [pool.apply_async(prepare_chunk, ((seed_, s0, min(step, start + n - s0), mh,
                                                  tuple(i for i in skip if s0 <= i < s0 + step)),))
                for s0 in range(start, start + n, step)]

    def produce():
        try:
            pending = [submit(c) for c in chunks[:2]]
            for k in range(len(chunks)):
                parts = pending.pop(0)
                if k + 2 < len(chunks):
                    pending.append(submit(chunks[k + 2]))
                ready.put([x for p in parts for x in unpack_chunk(p.get())])
        except Exception as e:          # surfaced by the main loop
            err.append(e)
        ready.put(None)

    def consume():
        try:
            while True:
                got = done.get()
                if got is None:
                    break
                items, res = got
                writer.write(batch_rows(items, res, seed))
        except Exception as e:
            err.append(e)

    tp = threading.Thread(target=produce, daemon=True)
    tw = threading.Thread(target=consume, daemon=True)
    t0 = time.perf_counter()
    tp.start()
    tw.start()
    queued = collections.deque()          # items of the batches handed to run_batches, in order

    def batches():
        while True:
            items = ready.get()
            if items is None or err:
                return
            queued.append(items)
            yield [it[2] for it in items]

    byid = {}

    def stream_mols():                    # molecules in stream order, their items kept by index
        k = 0
        for ms in batches():
            for it in queued.popleft():
                byid[k] = it
                k += 1
                yield it[2]

    def results():
        if refill:
            from .refill import run_refill
            for ids, _, res in run_refill(stream_mols(), slots=batch, level=level, precision=precision,
                                          guess=guess, net=net, e_tol=e_tol, diis_tol=diis_tol):
                res["host_ms"] = {"scf": res["host_ms"]["iterate"]}
                yield [byid.pop(int(i)) for i in ids], res
        else:
            # run_batches builds each next plan on its worker thread once the current batch's ERI
            # work is queued, and reuses the engine memory from batch to batch
            for _, res in run_batches(batches(), level=level, precision=precision, guess=guess, net=net,
                                      gradient=gradient, e_tol=e_tol, diis_tol=diis_tol):
                yield queued.popleft(), res

    try:
        for items, res in results():
            h = res["host_ms"]
            stats["gpu_s"] += 1e-3 * (h.get("engine", 0.0) + h.get("prepare", 0.0) + h["scf"] + h.get("gradient", 0.0))
            its = res["iterations"]
            stats["iterations"].append(its)
            stats["converged"] += int((its > 0).sum())
            stats["batches"] += 1
            done.put((items, res))
    finally:
        done.put(None)
        tw.join()
        tp.join(timeout=60)
        pool.terminate()
        writer.close()
    if err:
        raise err[0]
    wall = time.perf_counter() - t0
    its = np.concatenate(stats["iterations"]) if stats["iterations"] else np.zeros(0)
    its_c = its[its > 0]
    return {"molecules": int(len(its)), "batch": batch, "wall_s": wall, "molecules_per_s": len(its) / wall,
            "gpu_s": stats["gpu_s"], "gpu_molecules_per_s": len(its) / max(stats["gpu_s"], 1e-9),
            "converged": stats["converged"],
            "p50_iterations": float(np.percentile(its_c, 50)) if len(its_c) else None,
            "p99_iterations": float(np.percentile(its_c, 99)) if len(its_c) else None,
            "mean_iterations": float(its_c.mean()) if len(its_c) else None,
            "workers": workers, "out": out, "format": fmt, "skipped_already_written": skipped}


def main(argv=None):
    ap = argparse.ArgumentParser(description="stream molecules through the batched B200 SCF")
    ap.add_argument("--n", type=int, default=200000, help="molecules to generate")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--level", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--guess", default="learned", choices=["learned", "minao"])
    ap.add_argument("--out", default=None, help="output file (.parquet or .csv.gz)")
    ap.add_argument("--format", default=None, choices=["parquet", "csv"])
    ap.add_argument("--workers", type=int, default=None)
    ap.add_argument("--gradient", action="store_true", help="also write each molecule's nuclear gradient")
    ap.add_argument("--resume", action="store_true", help="skip the molecules whose rows --out already holds")
    ap.add_argument("--refill", action="store_true", help="refill converged slots from the stream")
    a = ap.parse_args(argv)
    fmt = a.format or ("csv" if a.out and a.out.endswith((".csv", ".csv.gz", ".gz")) else "parquet")
    r = run_stream(a.n, batch=a.batch, seed=a.seed, level=a.level, precision=a.precision, guess=a.guess,
                   out=a.out, fmt=fmt, workers=a.workers, gradient=a.gradient, resume=a.resume, refill=a.refill)
    print(json.dumps(r))
    return r


if __name__ == "__main__":
    main()
