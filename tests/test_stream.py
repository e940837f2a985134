"""Streaming dataset generation: stream determinism, QM1B / reference row schemas, GPU stream."""
import numpy as np
import pytest
import torch

from b200dft.molgen import stream_chunk, stream_molecule
from b200dft.stream import QM1B_COLUMNS, RowWriter, batch_rows, run_stream
from b200dft.constants import HARTREE_TO_EV


def test_stream_is_chunking_independent():
    a = stream_chunk((7, 0, 6, 9))
    b = stream_chunk((7, 0, 3, 9)) + stream_chunk((7, 3, 3, 9))
    assert [x[1] for x in a] == [x[1] for x in b]
    assert a[4][1] == stream_molecule(7, 4)
    assert len({x[1] for x in a}) == 6


def _fake_result(items):
    n = len(items)
    mo = np.zeros((n, 72))
    for j, (_, _, m) in enumerate(items):
        nocc = m.nelectron // 2
        mo[j, :m.nao] = np.linspace(-10, 1, m.nao)
        mo[j, nocc - 1], mo[j, nocc] = -0.3, 0.1
    last5 = np.full((n, 5), np.nan)
    last5[:, :3] = -40.0 + np.arange(3) * 1e-7
    return dict(energy=torch.full((n,), -40.0, dtype=torch.float64), mo_energy=torch.from_numpy(mo),
                last5=torch.from_numpy(last5), iterations=torch.full((n,), 6, dtype=torch.int32),
                converged=torch.ones(n, dtype=torch.bool))


def test_rows_parquet_schema(tmp_path):
    pq = pytest.importorskip("pyarrow.parquet")
    items = stream_chunk((1, 0, 5, 4))
    cols = batch_rows(items, _fake_result(items), seed=1)
    path = str(tmp_path / "rows.parquet")
    w = RowWriter(path, "parquet")
    w.write(cols)
    w.write(cols)
    w.close()
    t = pq.read_table(path)
    assert t.num_rows == 10
    for c in QM1B_COLUMNS:
        assert c in t.column_names
    r = t.slice(0, 1).to_pylist()[0]
    m = items[0][2]
    assert r["atoms"] == "".join(m.symbols) and r["z"] == [int(z) for z in m.charges]
    assert r["N"] == m.nao and len(r["pos"]) == 3 * m.natm
    assert abs(r["energy"] - (-40.0 * HARTREE_TO_EV)) < 1e-9
    assert abs(r["y"] - 0.4 * HARTREE_TO_EV) < 1e-9
    assert abs(r["std"] - np.std((-40.0 + np.arange(3) * 1e-7) * HARTREE_TO_EV)) < 1e-12


def test_rows_with_gradient(tmp_path):
    """force labels: the batch's gradient rows (atoms back to back) split per molecule, written as
    a flattened list beside pos"""
    pq = pytest.importorskip("pyarrow.parquet")
    items = stream_chunk((3, 0, 4, 5))
    res = _fake_result(items)
    nat = sum(it[2].natm for it in items)
    res["gradient"] = torch.arange(3 * nat, dtype=torch.float64).reshape(nat, 3)
    cols = batch_rows(items, res, seed=3)
    a0 = 0
    for k, it in enumerate(items):
        n3 = 3 * it[2].natm
        assert cols["gradient"][k] == list(np.arange(3 * a0, 3 * a0 + n3, dtype=float))
        a0 += it[2].natm
    path = str(tmp_path / "g.parquet")
    w = RowWriter(path, "parquet")
    w.write(cols)
    w.close()
    r = pq.read_table(path).to_pylist()
    assert all(len(row["gradient"]) == len(row["pos"]) for row in r)
    assert "gradient" not in batch_rows(items, _fake_result(items), seed=3)


def test_rows_csv_schema(tmp_path):
    import pandas as pd
    items = stream_chunk((2, 0, 3, 3))
    cols = batch_rows(items, _fake_result(items), seed=2)
    path = str(tmp_path / "data.csv")
    w = RowWriter(path, "csv")
    w.write(cols)
    w.write(cols)
    w.close()
    df = pd.read_csv(path, compression="gzip")
    assert len(df) == 6
    for c in ("smile", "atoms", "atom_positions", "energies", "std", "homo", "lumo", "hlgap", "N", "basis"):
        assert c in df.columns


@pytest.mark.gpu
def test_stream_gpu_matches_direct_batches(tmp_path):
    pq = pytest.importorskip("pyarrow.parquet")
    from b200dft.engine import RKSEngine
    path = str(tmp_path / "s.parquet")
    r = run_stream(40, batch=16, seed=3, guess="minao", out=path, workers=2, max_heavy=5)
    assert r["molecules"] == 40 and r["converged"] == 40
    assert r["p50_iterations"] is not None and r["p99_iterations"] >= r["p50_iterations"]
    t = pq.read_table(path).to_pydict()
    assert len(t["energy"]) == 40
    # the same molecules in one batch of 40 give the same energies
    items = stream_chunk((3, 0, 40, 5))
    eng = RKSEngine([m for _, _, m in items], level=0, precision="mixed", guess="minao")
    E = eng.run_converged()["energy"].cpu().numpy() * HARTREE_TO_EV
    eng.close()
    np.testing.assert_allclose(np.array(t["energy"]), E, atol=2e-3)   # eV, 1e-4 Ha


@pytest.mark.gpu
def test_stream_rows_match_fp64_oracle(tmp_path):
    """energies written by the stream (learned guess, mixed precision, slot refill) against the
    FP64 oracle SCF of the same molecules (20 fixed iterations, MINAO guess) at 1e-4 Ha"""
    pq = pytest.importorskip("pyarrow.parquet")
    from oracle import eri as oeri, rks
    from b200dft.engine import HostSetup
    path = str(tmp_path / "o.parquet")
    r = run_stream(24, batch=8, seed=5, out=path, workers=2, max_heavy=3, refill=True)
    assert r["molecules"] == 24 and r["converged"] == 24
    t = pq.read_table(path).to_pydict()
    rows = {int(sm.split(":")[2]): e for sm, e in zip(t["smile"], t["energy"])}   # gen:<seed>:<index>:..
    items = stream_chunk((5, 0, 24, 3))
    for k in (0, 7, 15, 23):
        i, _, m = items[k]
        s = HostSetup(m, 0)
        o = rks.scf(s.S, s.T, s.V, s.D0, oeri.eri_s8(m), rks.ao_values(m, s.coords), s.weights,
                    m.nelectron // 2, s.E_nuc, its=20)
        e_ref = o["energies"][-1, 0] * HARTREE_TO_EV
        assert abs(rows[i] - e_ref) <= 1e-4 * HARTREE_TO_EV, (k, rows[i], e_ref)


@pytest.mark.gpu
def test_run_batches_prefetch_matches_serial():
    """the public batch API gives the same results with the next plan built on a worker thread
    (overlapping the current batch) as without, and as one engine per batch"""
    from b200dft.engine import RKSEngine, run_batches
    b1 = [m for _, _, m in stream_chunk((5, 0, 12, 4))]
    b2 = [m for _, _, m in stream_chunk((5, 12, 9, 5))]
    pre = list(run_batches([b1, b2], guess="minao", prefetch=True))
    ser = list(run_batches([b1, b2], guess="minao", prefetch=False))
    assert [len(m) for m, _ in pre] == [12, 9]
    for (_, a), (_, b) in zip(pre, ser):
        # float32 atomics in the grid reductions: runs agree to rounding, not bit for bit
        np.testing.assert_allclose(a["energy"], b["energy"], rtol=0, atol=1e-9)
        np.testing.assert_array_equal(a["iterations"], b["iterations"])
        assert a["converged"].all() and a["h2d_bytes"] > 0
    eng = RKSEngine(b2, level=0, precision="mixed", guess="minao")
    E = eng.run_converged()["energy"].cpu().numpy()
    eng.close()
    np.testing.assert_allclose(pre[1][1]["energy"], E, rtol=0, atol=1e-9)


def _fake_engine(monkeypatch, fail_at=None):
    """run_batches with Plan and the per-batch SCF replaced by host stand-ins that record the
    order of events (no GPU)"""
    import threading
    from b200dft import engine
    log, lock = [], threading.Lock()

    class FakePlan:
        def __init__(self, mols):
            if fail_at is not None and mols[0] == fail_at:
                raise RuntimeError(f"plan {fail_at} failed")
            with lock:
                log.append(("plan", mols[0], threading.current_thread() is threading.main_thread()))
            self.first = mols[0]

    def fake_run_one(mols, plan, level, precision, guess, net, run_kw, after_prepare=None, gradient=False):
        assert plan.first == mols[0]
        with lock:
            log.append(("prepare", mols[0]))
        if after_prepare is not None:
            after_prepare()
        with lock:
            log.append(("scf", mols[0]))
        return {"energy": np.array([float(mols[0])]), "host_ms": {}, "kw": dict(run_kw), "gradient": gradient}

    monkeypatch.setattr(engine, "Plan", FakePlan)
    monkeypatch.setattr(engine, "_run_one", fake_run_one)
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 0)
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)
    return engine, log


@pytest.mark.parametrize("prefetch", [True, False])
def test_run_batches_order_and_prefetch_points(monkeypatch, prefetch):
    engine, log = _fake_engine(monkeypatch)
    batches = [[k, k] for k in range(5)]
    out = list(engine.run_batches(iter(batches), guess="minao", prefetch=prefetch, e_tol=1e-7))
    assert [m for m, _ in out] == batches                       # in order, one result per batch
    assert [float(r["energy"][0]) for _, r in out] == [0, 1, 2, 3, 4]
    # run_kw reaches each batch's SCF, with eager iterations unless the caller asks for a graph
    assert all(r["kw"] == {"e_tol": 1e-7, "graph": False} and "plan_wait" in r["host_ms"] for _, r in out)
    assert all(r["gradient"] is False for _, r in out)
    plans = [e for e in log if e[0] == "plan"]
    assert [e[1] for e in plans] == [0, 1, 2, 3, 4]
    assert plans[0][2]                                          # the first plan is made in place
    # with prefetch the later plans are made on the worker thread, each only after the previous
    # batch's setup and ERI work was queued; without it every plan is made on the caller's thread
    assert all(not e[2] for e in plans[1:]) if prefetch else all(e[2] for e in plans)
    for k in range(1, 5):
        assert log.index(("prepare", k - 1)) < log.index(plans[k])
        assert log.index(plans[k]) < log.index(("prepare", k))


def test_run_batches_passes_gradient(monkeypatch):
    engine, _ = _fake_engine(monkeypatch)
    out = list(engine.run_batches(iter([[0], [1]]), guess="minao", gradient=True, e_tol=1e-7))
    assert [r["gradient"] for _, r in out] == [True, True]
    assert out[0][1]["kw"] == {"e_tol": 1e-7, "graph": False}


def test_run_batches_empty_and_plan_errors(monkeypatch):
    engine, _ = _fake_engine(monkeypatch, fail_at=2)
    assert list(engine.run_batches(iter([]), guess="minao")) == []
    got = []
    with pytest.raises(RuntimeError, match="plan 2 failed"):
        for mols, _ in engine.run_batches(iter([[0], [1], [2], [3]]), guess="minao"):
            got.append(mols[0])
    assert got == [0, 1]     # the batches before the failing plan are all delivered


def test_packed_chunk_round_trip():
    """molecules sent packed between processes come back with identical arrays and accessors"""
    import pickle
    from b200dft.stream import prepare_chunk, unpack_chunk, static_columns
    args = (5, 0, 7, 6)
    ref = stream_chunk(args)
    got = unpack_chunk(pickle.loads(pickle.dumps(prepare_chunk(args))))
    assert [g[0] for g in got] == [r[0] for r in ref] and [g[1] for g in got] == [r[1] for r in ref]
    for (i, s, m, st), (_, _, r) in zip(got, ref):
        for name in ("coords", "charges", "_atm", "_bas", "_env", "ao_loc"):
            np.testing.assert_array_equal(getattr(m, name), getattr(r, name))
        assert (m.symbols, m.natm, m.nbas, m.nao, m.nelectron, m.basis, m.charge) == \
            (r.symbols, r.natm, r.nbas, r.nao, r.nelectron, r.basis, r.charge)
        assert m.energy_nuc() == r.energy_nuc() and st == static_columns(i, r, args[0])


def _stub_run_batches(batches, **kw):
    for mols in batches:
        n = len(mols)
        mo = np.zeros((n, 72))
        mo[:, :2] = [-0.5, 0.1]
        yield mols, {"energy": np.full(n, -40.0), "iterations": np.full(n, 6, np.int32),
                     "converged": np.ones(n, bool), "mo_energy": mo, "last5": np.full((n, 5), -40.0),
                     "diis_err": np.zeros(n), "its_run": 6, "host_ms": {"engine": 0.0, "prepare": 0.0, "scf": 0.0}}


@pytest.mark.parametrize("fmt", ["parquet", "csv"])
def test_stream_resume_skips_written_molecules(tmp_path, monkeypatch, fmt):
    """the engine stubbed out: a stream stopped after 7 molecules and resumed to 12 writes every
    molecule once (dft.py:247-283, -resume)"""
    import pandas as pd
    from b200dft import stream
    monkeypatch.setattr(stream, "run_batches", _stub_run_batches)
    path = str(tmp_path / ("rows.parquet" if fmt == "parquet" else "rows.csv.gz"))
    kw = dict(batch=5, seed=3, guess="minao", out=path, fmt=fmt, workers=2)
    r1 = stream.run_stream(7, **kw)
    assert r1["molecules"] == 7 and r1["skipped_already_written"] == 0
    r2 = stream.run_stream(12, resume=True, **kw)
    assert r2["molecules"] == 5 and r2["skipped_already_written"] == 7
    if fmt == "parquet":
        smiles = pd.read_parquet(path)["smile"].tolist()
    else:
        smiles = pd.read_csv(path, compression="gzip")["smile"].tolist()
    assert sorted(int(s.split(":")[2]) for s in smiles) == list(range(12))
    assert stream.done_indices(path, fmt, 3) == set(range(12)) and stream.done_indices(path, fmt, 4) == set()
    r3 = stream.run_stream(12, resume=True, **kw)            # nothing left to do
    assert r3["molecules"] == 0 and r3["skipped_already_written"] == 12


@pytest.mark.gpu
def test_stream_force_labels_match_engine(tmp_path):
    """force labels (run_stream(gradient=True)): each row's gradient equals the batched engine's
    gradient of the same molecule (float64 SCF, the same two batches run directly)"""
    pq = pytest.importorskip("pyarrow.parquet")
    from b200dft.engine import RKSEngine
    path = str(tmp_path / "f.parquet")
    r = run_stream(12, batch=6, seed=5, guess="minao", precision="fp64", out=path, workers=2, max_heavy=4,
                   gradient=True)
    assert r["molecules"] == 12 and r["converged"] == 12
    t = pq.read_table(path).to_pydict()
    mols, gs = [], []
    for start in (0, 6):                      # the stream's two batches, run directly
        mb = [m for _, _, m in stream_chunk((5, start, 6, 4))]
        eng = RKSEngine(mb, level=0, precision="fp64", guess="minao")
        eng.run_converged()
        gs.append(eng.gradient().cpu().numpy())
        eng.close()
        mols += mb
    g = np.concatenate(gs)
    a0 = 0
    for k, m in enumerate(mols):
        assert len(t["gradient"][k]) == 3 * m.natm
        np.testing.assert_allclose(np.array(t["gradient"][k]).reshape(-1, 3), g[a0:a0 + m.natm], atol=1e-6, rtol=0)
        a0 += m.natm


def _stub_run_refill(mols, slots=4, **kw):
    """retires molecules out of stream order (every other slot first), like a refill would"""
    buf, k = [], 0
    for m in mols:
        buf.append((k, m))
        k += 1
    order = buf[1::2] + buf[0::2]
    for s in range(0, len(order), 3):
        part = order[s:s + 3]
        n = len(part)
        mo = np.zeros((n, 72))
        mo[:, :2] = [-0.5, 0.1]
        e = np.array([-40.0 - i for i, _ in part])
        yield np.array([i for i, _ in part]), [m for _, m in part], {
            "energy": e, "iterations": np.full(n, 6, np.int32), "converged": np.ones(n, bool), "mo_energy": mo,
            "last5": np.repeat(e[:, None], 5, 1), "diis_err": np.zeros(n), "its_run": 6,
            "host_ms": {"iterate": 0.0}}


def test_stream_refill_rows_follow_their_molecules(tmp_path, monkeypatch):
    """with slot refill the results come back out of order; each row still carries its own
    molecule's result"""
    import pandas as pd
    from b200dft import refill, stream
    monkeypatch.setattr(refill, "run_refill", _stub_run_refill)
    path = str(tmp_path / "rows.parquet")
    r = stream.run_stream(11, batch=4, seed=3, guess="minao", out=path, workers=2, refill=True)
    assert r["molecules"] == 11 and r["converged"] == 11
    t = pd.read_parquet(path)
    idx = [int(s.split(":")[2]) for s in t["smile"]]
    assert sorted(idx) == list(range(11)) and idx != list(range(11))
    np.testing.assert_allclose(t["energy"].to_numpy(), (-40.0 - np.array(idx)) * 27.2114079527)
