"""Batched SCF with slot refill: converged molecules retire and new molecules of the stream take
their slots while the others keep iterating.

``run_batches`` (engine.py) holds a batch until its slowest molecule has converged, so the last
iterations of every batch run with most slots empty.  Here a batch of ``slots`` molecules
iterates (the SCF step of ``RKSEngine.run_converged``: eager launches, or with ``graph`` one
captured CUDA graph replayed per iteration) until at most ``refill_at`` of them are still active;
then

  * the molecules that converged (or reached ``max_its``) retire: their results go to the host;
  * the molecules still iterating are carried into a new plan, first, with their whole SCF state
    -- density, J / K / V_xc, Fock matrix, DIIS error and Fock rings and B matrix, eigenvector
    warm start, orbital energies, iteration counters, the last five energies, the fallback
    flags -- and their s8 and exchange lists copied on the device (b2_copy_blocks), so they
    continue exactly where they were;
  * new molecules from the stream fill the remaining slots: device setup, ERIs (their own plan,
    then copied into place), the learned guess with its MINAO fallback, and the first XC and
    J/K of their initial density.

The reference's counterpart is its conformer loop (dft.py:236-691), which runs one molecule at a
time and has no batching to refill.  Each molecule follows the same iteration sequence as in
``run_converged``, so its result does not depend on which slots it shared with whom.
"""
import time

import numpy as np
import torch

from ._lib import lib, check, ptr, stream_handle
from .engine import RKSEngine, Plan, NMO

# per-molecule state arrays of RKSEngine: (attribute, elements per molecule kind)
_MAT = ("D", "J", "K", "Vxc", "H", "diffJK", "C", "eig_ws")      # n_mat layout, nao^2 each
_RING = ("ring_err", "ring_h")                                   # 9 nao^2 each at 9 mat_off
_PERMOL = (("diis_err", 1), ("exc", 1), ("energy", 5), ("mo_energy", NMO), ("bmat", 100),
           ("iter", 1), ("sweeps", 1))


def _spans(off, size, sel):
    """concatenated index ranges [off[m], off[m] + size[m]) for m in sel"""
    sel = np.asarray(sel, np.int64)
    if len(sel) == 0:
        return np.zeros(0, np.int64)
    o = np.asarray(off, np.int64)[sel]
    n = np.asarray(size, np.int64)[sel]
    first = np.cumsum(n) - n                           # position of each range in the result
    return np.repeat(o - first, n) + np.arange(int(n.sum()), dtype=np.int64)


class _Runner:
    """one engine (one plan) plus the host-side convergence bookkeeping of its molecules"""

    def __init__(self, eng, ids, fallback):
        self.eng = eng
        self.ids = np.asarray(ids, np.int64)           # stream index of each slot's molecule
        nm = len(ids)
        dev = eng.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.e_prev = torch.full((nm,), float("inf"), **f64)
        self.err_prev = torch.full((nm,), float("inf"), **f64)
        self.hist = torch.full((nm, 5), float("nan"), **f64)
        self.conv_it = torch.full((nm,), -1, dtype=torch.int32, device=dev)
        self.its = torch.zeros(nm, dtype=torch.int32, device=dev)        # iterations since the start
        self.fell_back = torch.zeros(nm, dtype=torch.bool, device=dev)
        self.use_fb = fallback and eng.D0_minao is not None
        self.graph = None
        self.keep = None                                  # buffers of queued work (released later)


def _carry(old, new, sel, nsel):
    """copy the SCF state of old-slot molecules ``sel`` into new slots 0..len(sel)-1"""
    eo, en = old.eng, new.eng
    Po, Pn = eo.plan, en.plan
    nao_o = Po.nao.astype(np.int64)
    src = torch.from_numpy(_spans(Po.mat_off, nao_o ** 2, sel)).to(eo.device)
    dst = torch.from_numpy(_spans(Pn.mat_off, Pn.nao.astype(np.int64) ** 2, nsel)).to(eo.device)
    for a in _MAT:
        getattr(en, a)[dst] = getattr(eo, a)[src]
    src9 = torch.from_numpy(_spans(9 * Po.mat_off, 9 * nao_o ** 2, sel)).to(eo.device)
    dst9 = torch.from_numpy(_spans(9 * Pn.mat_off, 9 * Pn.nao.astype(np.int64) ** 2, nsel)).to(eo.device)
    for a in _RING:
        getattr(en, a)[dst9] = getattr(eo, a)[src9]
    s_t = torch.from_numpy(np.asarray(sel, np.int64)).to(eo.device)
    d_t = torch.from_numpy(np.asarray(nsel, np.int64)).to(eo.device)
    for a, k in _PERMOL:
        o, n = getattr(eo, a).view(Po.nmol, k), getattr(en, a).view(Pn.nmol, k)
        n[d_t] = o[s_t]
    for a in ("e_prev", "err_prev", "hist", "conv_it", "its", "fell_back"):
        getattr(new, a)[d_t] = getattr(old, a)[s_t]
    en.active[d_t] = eo.active[s_t]
    # s8 and exchange lists: one block per molecule, bytes
    es = en.eri.element_size()
    n4 = np.array([(n * (n + 1) // 2) * (n * (n + 1) // 2 + 1) // 2 for n in nao_o[sel]], np.int64)
    offs = torch.from_numpy(np.stack([Po.eri_off[sel] * es, Pn.eri_off[nsel] * es, n4 * es]).astype(np.int64)).to(eo.device)
    for a in ("eri", "eri_x"):
        check(lib().b2_copy_blocks(len(sel), ptr(getattr(eo, a)), ptr(getattr(en, a)), ptr(offs[0]), ptr(offs[1]),
                                   ptr(offs[2]), stream_handle()), "b2_copy_blocks")


def _fill_eri(eng, new_slots, mols):
    """s8 and exchange lists of the new molecules: computed on their own plan, copied into place.
    Returns what must outlive the queued work (the plan and its buffers): the caller keeps it
    until a later synchronisation."""
    if not new_slots:
        return None
    P = Plan(mols)
    dt = eng.eri.dtype
    tmp = torch.empty(max(1, P.n_eri), dtype=dt, device=eng.device)
    tmpx = torch.empty_like(tmp)
    check(lib().b2_eri_s8(P.h, eng.prec, ptr(tmp), stream_handle()), "b2_eri_s8")
    if eng.eri_threshold > 0.0:
        check(lib().b2_eri_threshold(P.h, eng.prec, ptr(tmp), eng.eri_threshold, stream_handle()),
              "b2_eri_threshold")
    check(lib().b2_jk_exchange(P.h, eng.prec, ptr(tmp), ptr(tmpx), stream_handle()), "b2_jk_exchange")
    es = tmp.element_size()
    nao = P.nao.astype(np.int64)
    n4 = (nao * (nao + 1) // 2) * (nao * (nao + 1) // 2 + 1) // 2
    offs = torch.from_numpy(np.stack([P.eri_off * es, eng.plan.eri_off[new_slots] * es, n4 * es])
                            .astype(np.int64)).to(eng.device)
    for src, dst in ((tmp, eng.eri), (tmpx, eng.eri_x)):
        check(lib().b2_copy_blocks(len(new_slots), ptr(src), ptr(dst), ptr(offs[0]), ptr(offs[1]),
                                   ptr(offs[2]), stream_handle()), "b2_copy_blocks")
    return P, tmp, tmpx, offs


def _start(mols, ids, carried, level, precision, guess, net, fallback, eri_threshold):
    """engine for ``mols`` (the carried molecules first, then new ones) with the carried state in
    place and the new molecules initialised"""
    nc = 0 if carried is None else len(carried[1])
    # every refill allocates lists of a new size: hand torch's cached blocks back to the driver
    # when they hold most of the device (the plan tables allocate outside torch's cache)
    free, total = torch.cuda.mem_get_info()
    if free < 0.3 * total:
        torch.cuda.empty_cache()
    eng = RKSEngine(mols, level=level, precision=precision, guess=guess, net=net, eri_threshold=eri_threshold)
    # GPU work first (setup, the new molecules' ERIs), then the host work of the learned guess and
    # of the carry, which overlaps it
    eng.device_setup()
    new_slots = list(range(nc, len(mols)))
    keep = _fill_eri(eng, new_slots, mols[nc:])
    eng._eri_done = True
    eng._start_guess()
    if eng._guess_done is not None:
        torch.cuda.current_stream(eng.device).wait_event(eng._guess_done)
        eng._guess_done = None
    r = _Runner(eng, ids, fallback)
    r.keep = keep
    eng.D.copy_(eng.D0)
    eng.iter.zero_()
    eng.active.fill_(1)
    if carried is not None:
        old, sel = carried
        _carry(old, r, sel, list(range(nc)))
    newmask = torch.zeros(len(mols), dtype=torch.int32, device=eng.device)
    newmask[nc:] = 1
    eng.scf_xc(active=newmask)
    eng.jk(active=newmask)
    return r


def _capture(r, use_diis):
    eng = r.eng
    st = torch.cuda.Stream()
    st.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(st):
        g.capture_begin(capture_error_mode="thread_local")
        try:
            eng.step(use_diis)
        finally:
            g.capture_end()
    torch.cuda.current_stream().wait_stream(st)
    r.graph = g


def _iterate(r, stop_at, max_its, e_tol, diis_tol, use_diis, rise, fallback_window, graph=False):
    """iterate (eager steps, or graph replays) until at most ``stop_at`` molecules are active;
    molecules that reach ``max_its`` stop as unconverged"""
    eng = r.eng
    nm = eng.plan.nmol
    its_run = 0
    while True:
        n_act = int(eng.active.sum().item())
        if n_act == 0 or n_act <= stop_at:
            return its_run
        if graph:
            if r.graph is None:
                _capture(r, use_diis)
            r.graph.replay()
            eng.graph_replays += 1
        else:
            eng.step(use_diis)
        its_run += 1
        act = eng.active > 0
        e = eng.energy.view(nm, 5)[:, 0]
        r.its += act.to(torch.int32)
        slot = (r.its - 1).remainder(5).to(torch.int64).clamp(min=0)
        cur = r.hist.gather(1, slot[:, None])[:, 0]
        r.hist.scatter_(1, slot[:, None], torch.where(act, e, cur)[:, None])
        newly = act & ((e - r.e_prev).abs() < e_tol) & (eng.diis_err < diis_tol)
        r.conv_it = torch.where(newly, r.its, r.conv_it)
        eng.active.masked_fill_(newly | (r.its >= max_its), 0)
        r.e_prev = torch.where(eng.active > 0, e, r.e_prev)
        if r.use_fb:
            err = eng.diis_err
            bad = ((eng.active > 0) & ~r.fell_back & (eng.iter >= 2) & (eng.iter <= fallback_window)
                   & (err > rise * r.err_prev))
            r.err_prev = torch.where(eng.active > 0, err, r.err_prev)
            if bool(bad.any()):
                eng._restart_from_minao(bad)
                r.fell_back |= bad
                r.e_prev = torch.where(bad, torch.full_like(r.e_prev, float("inf")), r.e_prev)
                r.err_prev = torch.where(bad, torch.full_like(r.err_prev, float("inf")), r.err_prev)


def _retire(r, mols_by_id, done_mask):
    """host results of the slots in ``done_mask`` (numpy bool)"""
    eng = r.eng
    nm = eng.plan.nmol
    sel = np.nonzero(done_mask)[0]
    if len(sel) == 0:
        return None
    t = torch.from_numpy(sel.astype(np.int64)).to(eng.device)
    conv = r.conv_it[t].cpu().numpy()
    its = r.its[t].cpu().numpy()
    hist = r.hist[t].cpu().numpy()
    # last five energies, oldest first (the ring slot of iteration k is (k - 1) mod 5)
    order = [(its - 5 + k).clip(min=0) % 5 for k in range(5)]
    last5 = np.stack([hist[np.arange(len(sel)), o] for o in order], 1)
    last5[np.arange(5)[None, :] < 5 - its[:, None]] = np.nan
    out = {"energy": eng.energy.view(nm, 5)[t, 0].cpu().numpy(),
           "iterations": np.where(conv > 0, conv, -1).astype(np.int32),
           "converged": conv > 0,
           "mo_energy": eng.mo_energy.view(nm, NMO)[t].cpu().numpy(),
           "diis_err": eng.diis_err[t].cpu().numpy(), "last5": last5,
           "fell_back": r.fell_back[t].cpu().numpy(), "its_run": int(its.max())}
    ids = r.ids[sel]
    return ids, [mols_by_id.pop(int(i)) for i in ids], out


def run_refill(molecules, slots=4096, level=0, precision="mixed", guess="learned", net=None,
               refill_at=0.3, max_its=40, e_tol=1e-6, diis_tol=1e-4, use_diis=True, fallback=True,
               rise=3.0, fallback_window=5, eri_threshold=0.0, graph=False):
    """SCF of every molecule of the iterable ``molecules`` with ``slots`` molecules resident on
    the GPU at a time; whenever at most ``refill_at`` of the slots are still iterating, the
    retired slots are refilled from the stream.  Yields ``(ids, mols, result)`` per refill:
    stream indices, molecules and host arrays of the retired molecules (energy, iterations
    (-1: not converged within ``max_its``), converged, mo_energy, diis_err, last5, fell_back,
    its_run, host_ms).  Every refill makes a new plan, so the SCF steps run eager unless ``graph``
    (a captured graph then serves one plan's iterations)."""
    if guess == "learned" and net is None:
        from .train_guess import load
        net = load()
    it = iter(molecules)
    next_id = 0
    mols_by_id = {}

    def take(n):
        nonlocal next_id
        got = []
        for _ in range(n):
            m = next(it, None)
            if m is None:
                break
            mols_by_id[next_id] = m
            got.append((next_id, m))
            next_id += 1
        return got

    t0 = time.perf_counter()
    first = take(slots)
    if not first:
        return
    r = _start([m for _, m in first], [i for i, _ in first], None, level, precision, guess, net,
               fallback, eri_threshold)
    exhausted = len(first) < slots
    while True:
        th = time.perf_counter()
        # once the stream is exhausted, the survivors still move to smaller plans (no new
        # molecules) so the last iterations launch only their work; small batches drain in place
        nm = r.eng.plan.nmol
        stop_at = int(refill_at * (nm if exhausted else slots)) if (not exhausted or nm > 64) else -1
        n = _iterate(r, stop_at, max_its, e_tol, diis_tol, use_diis, rise, fallback_window, graph)
        t_iter = time.perf_counter() - th
        act = r.eng.active.cpu().numpy() > 0
        got = _retire(r, mols_by_id, ~act)
        if got is not None:
            ids, ms, out = got
            out["host_ms"] = {"iterate": 1e3 * t_iter, "iterations": n, "since_start": 1e3 * (time.perf_counter() - t0)}
            yield ids, ms, out
        survivors = np.nonzero(act)[0]
        if exhausted and len(survivors) == 0:
            break
        fresh = [] if exhausted else take(slots - len(survivors))
        exhausted = exhausted or len(fresh) < slots - len(survivors)
        if len(survivors) == 0 and not fresh:
            break
        mols = [mols_by_id[int(r.ids[s])] for s in survivors] + [m for _, m in fresh]
        ids = [int(r.ids[s]) for s in survivors] + [i for i, _ in fresh]
        r.keep = None            # its ERI plan's work finished long ago (iterations synchronised since)
        old = r
        r = _start(mols, ids, (old, survivors), level, precision, guess, net, fallback, eri_threshold)
        old.graph = None
        old.eng.close()
        del old
    r.eng.close()
