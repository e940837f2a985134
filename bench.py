"""Benchmark: SCF molecules/s on one B200 (batched mixed-precision engine).

Workload: a seeded batch of synthetic molecules with the shape of the batched
configuration (1-9 heavy atoms from C/N/O/F = 0.7/0.1/0.15/0.05, H to valence, STO-3G,
B3LYP, level-0 grid); synthetic because the reference's GDB/QM1B data is not available.
One step = the whole hot path over the batch from inputs resident in HBM: device setup
(1e matrices, Becke grid, MINAO guess, L), the learned initial guess (network forward pass;
MINAO is the per-molecule fallback), ERIs (FP32, s8), and the SCF iterated per molecule until
|dE| < 1e-6 Ha and DIIS error < 1e-4 with converged molecules retired.
``e2e`` runs the same through the public API from host buffers (plan creation from the
libcint host arrays, host->device copies, results copied back).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--nmol M] [--impl b200|reference]
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# the legs allocate engines of many sizes one after another: let torch's allocator grow and
# shrink its segments instead of caching one block per size
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")
sys.path.insert(0, os.path.join(ROOT, "pyscf-ipu_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "SCF molecules/s on 1 B200 at |dE|<=0.1 mHa: batched+learned vs plain FP64"
UNIT = "molecules/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def _tensor_peak(sustained=True):
    """bf16 dense peak: the sustained figure for a kernel timed inside a long step, the burst
    figure for a kernel timed alone"""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if sustained and "bf16_tflops_sustained" in d:
            return d["bf16_tflops_sustained"], "measured sustained"
        return d.get("bf16_tflops", 1590.0), "measured burst"
    return (1400.0, "fallback sustained") if sustained else (1590.0, "fallback burst")


def quartet_counts(mols):
    """canonical shell quartets (IJ >= KL over shell pairs I >= J) of the molecules and their
    primitive quartets before screening"""
    quartets = prim = 0
    for m in mols:
        npr = np.asarray(m._bas)[:, 2].astype(np.int64)            # libcint NPRIM_OF slot
        pp = (npr[:, None] * npr[None, :])[np.tril_indices(len(npr))]
        s = int(pp.sum())
        quartets += len(pp) * (len(pp) + 1) // 2
        prim += (s * s + int((pp * pp).sum())) // 2
    return quartets, prim


def _timed(fn, n):
    """mean CUDA-event time (ms) of n calls on the current stream, after one warm-up call"""
    import torch
    fn()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(n):
        fn()
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / n


def kernel_rooflines(eng, precision):
    """Roofline figures of the three kernel families on the resident batch, each timed with
    CUDA events around repeated calls of the entry the SCF uses (after the timed region, same
    batch and data):
      * XC (k_xc_tq, tensor bound): algorithmic flops 4 G N^2 per molecule (the rho and V_xc
        contractions, N = nao unpadded) against the measured burst bf16 dense peak (the calls are
        timed alone, back to back); the operands are split tf32 (nominal tf32 rate = half the
        bf16 rate).
      * J/K (k_symv, HBM bound): algorithmic bytes n4 x 4 B per molecule (the s8 list read once,
        D/J/K on chip) against the measured HBM copy rate.
      * ERI (k_eri_*, float32 SIMT): shell and primitive quartets per second.
    Returns the list, dominant kernel (largest device-time share) first."""
    from b200dft._lib import lib, check, ptr, stream_handle
    P = eng.plan
    hbm, hbm_kind = _peaks()
    tpk, tkind = _tensor_peak(sustained=False)     # the kernel is timed alone (back-to-back calls)
    rbytes = 4 if precision == "mixed" else 8
    out = []
    G = np.diff(P.grid_off).astype(np.float64)
    N = P.nao.astype(np.float64)
    flops = float((4.0 * G * N * N).sum())
    xc_ms = _timed(lambda: eng.xc(active=None), 5)
    tf = flops / (xc_ms / 1e3) / 1e12
    # DRAM bytes per launch: the ncu capture of the NB = 64 bucket's launch on the 512-molecule
    # batch (57.83 MB read + 0.19 MB written for 1 601 800 grid points: 36.2 B per point, the
    # point's coordinates and weight plus its share of D and V), scaled by the batch's points
    xc_traffic = 36.22 * float(G.sum()) if precision == "mixed" else None
    out.append({"kernel": "k_xc_tq (per-bucket persistent)" if precision == "mixed" else "k_xc_direct",
                "bound": "tensor",
                "achieved": tf, "peak": tpk, "unit": "TFLOP/s", "frac": tf / tpk, "traffic": xc_traffic,
                "peak_kind": f"{tkind} bf16 dense (of measured)", "algorithmic_flops_per_launch": flops,
                "ms_per_launch": xc_ms, "operands": "split tf32, fp32 accumulate"})
    eng.D.copy_(eng.D0)
    jk_ms = _timed(lambda: eng.jk(active=None), 10)
    n4 = float(sum(int(n) * (int(n) + 1) // 2 * (int(n) * (int(n) + 1) // 2 + 1) // 2 for n in P.nao))
    jk_bytes = n4 * rbytes
    gbs = jk_bytes / (jk_ms / 1e3) / 1e9
    read = (2 if eng.jk_impl == "pairs" else 1) * P.n_eri * rbytes
    # DRAM bytes per launch: ncu capture of k_symv on the 256-molecule batch (868.8 MB read +
    # 6.4 MB written for 860.7 MB of float32 list entries in both lists), scaled by list size
    traffic = read * (875.2 / 860.7) if (precision == "mixed" and eng.jk_impl == "pairs") else None
    out.append({"kernel": "k_symv" if eng.jk_impl == "pairs" else "k_jk_s8", "bound": "hbm", "achieved": gbs,
                "peak": hbm, "unit": "GB/s", "frac": gbs / hbm, "traffic": traffic,
                "peak_kind": f"{hbm_kind} HBM copy", "algorithmic_bytes_per_launch": jk_bytes,
                "bytes_read_per_launch": read, "ms_per_launch": jk_ms})
    quartets, prim = quartet_counts(eng.mols)
    prec = 64 if precision == "fp64" else 32
    eri_ms = _timed(lambda: check(lib().b2_eri_s8(P.h, prec, ptr(eng.eri), stream_handle()), "b2_eri_s8"), 3)
    e = {"kernel": "k_eri_fl / k_eri_sq (16 class kernels)", "bound": "fp32 simt", "ms_per_launch": eri_ms,
         "shell_quartets_per_s": quartets / (eri_ms / 1e3), "shell_quartets": quartets,
         "primitive_quartets_unscreened": prim}
    if prec == 32:
        # evaluated primitive quartets and their arithmetic by the per-class counts of
        # csrc/eri_flops.h (generated from the kernels' own code), against the FP32 FMA rate
        # measured on this GPU by the library's microbenchmark
        work = np.zeros(3)
        pk = ctypes.c_double(0.0)
        check(lib().b2_eri_work(P.h, ptr(work)), "b2_eri_work")
        check(lib().b2_fp32_peak(ctypes.byref(pk)), "b2_fp32_peak")
        tf = work[1] / (eri_ms / 1e3) / 1e12
        e.update({"achieved": tf, "peak": pk.value, "unit": "TFLOP/s", "frac": tf / pk.value,
                  "peak_kind": "measured FP32 FMA (b2_fp32_peak)", "primitive_quartets": work[0],
                  "algorithmic_flops_per_launch": work[1], "special_ops_per_launch": work[2],
                  "primitive_quartets_per_s": work[0] / (eri_ms / 1e3)})
    out.append(e)
    return out


class Clocks:
    """nvidia-smi sampler during the timed region."""

    def __init__(self):
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            idx = os.environ.get("LOCAL_RANK", "0")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", idx, f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(2)
        except Exception:
            self.proc.kill()
        sm = [float(s[0]) for s in self.samples if s and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) > 1 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, n in enumerate(names):
            if any(len(s) > 3 + k and s[3 + k].lower().startswith("active") for s in self.samples):
                reasons.append(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def molecules(nmol, seed):
    from b200dft.molgen import config3_batch
    from b200dft.mole import Mole
    return [Mole(s) for s in config3_batch(nmol, seed=seed)]


# ------------------------------------------------------------------ CPU oracle baseline
def _oracle_one(args):
    atom, level, use_ref = args
    import os as _os
    import sys as _sys
    _sys.path.insert(0, _os.path.join(ROOT, "pyscf-ipu_b200"))
    _sys.path.insert(0, ROOT)
    from oracle import eri as oeri, rks
    from b200dft.mole import Mole
    from b200dft.engine import HostSetup
    m = Mole(atom)
    s = HostSetup(m, level)
    s8 = oeri.ref_eri_s8(m) if use_ref else oeri.eri_s8(m)
    ao = rks.ao_values(m, s.coords)
    r = rks.scf(s.S, s.T, s.V, s.D0, s8, ao, s.weights, m.nelectron // 2, s.E_nuc, its=20)
    return float(r["energies"][-1, 0])


def _cpu_pool(procs, level, use_ref):
    """spawned worker processes, one BLAS thread each (one molecule per process is the
    throughput layout), started and warmed up (modules imported, one small SCF each) before any
    timing"""
    import multiprocessing as mp
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"                  # inherited by the spawned workers' numpy
    pool = mp.get_context("spawn").Pool(procs)
    pool.map(_oracle_one, [("H 0 0 0; H 0 0 0.74", level, use_ref)] * procs, chunksize=1)
    return pool


def cpu_baseline(atoms, level, use_ref, pool=None):
    """CPU-path SCF throughput on ``atoms``: on the worker pool, or in this process on one
    BLAS thread (the one-core baseline)"""
    t0 = time.perf_counter()
    if pool is not None:
        es = pool.map(_oracle_one, [(a, level, use_ref) for a in atoms], chunksize=1)
    else:
        from threadpoolctl import threadpool_limits
        with threadpool_limits(1):
            es = [_oracle_one((a, level, use_ref)) for a in atoms]
    dt = time.perf_counter() - t0
    return len(atoms) / dt, dt, es


def run_reference(a):
    """--impl reference: the reference's CPU path (its own compiled int2e_sph for the ERIs,
    the FP64 port for the rest) on the host cores, bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import eri as oeri
    use_ref = oeri.ref_available()
    from b200dft.molgen import config3_batch
    procs = os.cpu_count() or 1
    per_step = max(procs, 8)
    atoms = config3_batch(per_step * (a.steps + a.warmup), seed=a.seed)
    vals = []
    t_all = 0.0
    pool = _cpu_pool(procs, a.level, use_ref)
    try:
        for k in range(a.warmup + a.steps):
            v, dt, _ = cpu_baseline(atoms[k * per_step:(k + 1) * per_step], a.level, use_ref, pool)
            if k >= a.warmup:
                vals.append(v)
                t_all += dt
    finally:
        pool.close()                     # workers exit normally (their loaded libraries stay visible)
        pool.join()
    value = float(np.mean(vals))
    kind = "reference" if use_ref else "port"
    sample = (f"{per_step} molecules per step of the batched distribution, 20 SCF iterations, level-{a.level} "
              f"grid; {procs} worker processes with one BLAS thread each, started before timing")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1000 * t_all / max(1, a.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": "batched uneven STO-3G B3LYP molecules (1-9 heavy atoms C/N/O/F), level-0 grid",
                   "nmol": per_step},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ------------------------------------------------------------------ B200 arm
def gradient_timing(mols, a, net):
    """Nuclear gradients (b2_grad) of a converged batch: CUDA-event time of the full gradient and
    of each term (one-electron, two-electron, exchange-correlation, nuclear), after one warm-up
    call; the orbitals and grid stay resident between calls."""
    import torch
    from b200dft.engine import RKSEngine
    eng = RKSEngine(mols, level=a.level, precision=a.precision, guess=a.guess, net=net)
    try:
        r = eng.run_converged()
        ms = {}
        for name, parts in (("full", 15), ("one_electron", 1), ("two_electron", 2), ("xc", 4), ("nuclear", 8)):
            eng.gradient(parts=parts)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            t0.record()
            for _ in range(3):
                eng.gradient(parts=parts)
            t1.record()
            torch.cuda.synchronize()
            ms[name] = t0.elapsed_time(t1) / 3
        return {"molecules": len(mols), "converged": int(r["converged"].sum().item()), "ms_per_call": ms,
                "molecules_per_s": len(mols) / (ms["full"] / 1000.0), "dtype": "f64",
                "timing": "CUDA events, mean of 3 calls after one warm-up call"}
    finally:
        eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--nmol", type=int, default=4096)
    ap.add_argument("--level", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--guess", default="learned", choices=["learned", "minao"])
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--cpu-sample", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-mode", action="store_true", help="timed steps only (for ncu captures)")
    ap.add_argument("--stream", type=int, default=204800,
                    help="streaming leg: molecules through the public stream API with slot refill (0: off)")
    ap.add_argument("--grad", type=int, default=None,
                    help="also time the nuclear gradient (b2_grad) of the first N converged molecules "
                         "(0: off; default 512, or off with --profile-mode)")
    ap.add_argument("--config2-only", action="store_true",
                    help="only the single-molecule level-3 report (for per-kernel ncu captures)")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference(a)
    if a.config2_only:
        print(json.dumps({"config2": config2_report()}))
        return None

    import torch
    import torch.distributed as dist
    from b200dft.engine import RKSEngine, Plan
    from b200dft._lib import launch_count
    from b200dft import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        if "WORLD_SIZE" in os.environ:
            sys.exit(f"bench.py: --gpus {a.gpus} but WORLD_SIZE={world}")
        return spawn_ranks(a.gpus)               # one process per GPU, as torchrun would start them
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return shard.max_over_ranks(x, world, device="cuda")

    # weak scaling: every rank runs its own shard of molecules (no data-path collective)
    mols = molecules(a.nmol, seed=shard.shard_seed(a.seed, rank))
    net = None
    if a.guess == "learned":
        from b200dft.train_guess import load
        net = load()
    eng = RKSEngine(mols, level=a.level, precision=a.precision, guess=a.guess, net=net)
    ev = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for k in ("setup", "eri", "ao", "scf")}

    def one_step(record=False):
        eng._setup_done = False
        eng._eri_done = False
        eng._ao_done = False
        if record:
            ev["setup"][0].record()
        eng.device_setup()
        if record:
            ev["setup"][1].record()
            ev["eri"][0].record()
        eng.compute_eri()
        if record:
            ev["eri"][1].record()
            ev["ao"][0].record()
            ev["ao"][1].record()
            ev["scf"][0].record()
        r = eng.run_converged()
        if record:
            ev["scf"][1].record()
        return r

    for _ in range(a.warmup):
        res = one_step()
    barrier()
    clk = Clocks()
    clk.start()
    phase = {k: 0.0 for k in ev}
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    barrier()
    eng.graph_replays = 0
    eng._captured = 0
    lc0 = launch_count()
    t_start.record()
    its_total = 0
    for _ in range(a.steps):
        res = one_step(record=True)
        its_total += res["its_run"]
        torch.cuda.synchronize()
        for k, (s, e) in ev.items():
            phase[k] += s.elapsed_time(e)
    t_end.record()
    barrier()
    clocks = clk.stop()
    gpu_launches = eng.kernels_launched(lc0)
    ms = max_over_ranks(t_start.elapsed_time(t_end)) / a.steps
    value = shard.aggregate_rate(a.nmol, world, ms / 1000.0)
    conv = res["converged"].cpu().numpy()
    iters = res["iterations"].cpu().numpy()
    res["D"] = eng.D.clone()                 # converged densities of the timed batch (parity)

    # ---- roofline figures of the kernel families (dominant first) on the resident batch
    rooflines = [{"note": "not measured (profile mode: timed steps only)"}]
    if not a.profile_mode:
        try:
            rooflines = kernel_rooflines(eng, a.precision)
        except Exception as e:  # noqa: BLE001  (recorded in the line, it does not void it)
            rooflines = [{"error": f"{type(e).__name__}: {e}"}]
    roofline = rooflines[0]

    grad = None
    if a.grad is None:
        a.grad = 0 if a.profile_mode else 512
    if a.grad > 0 and rank == 0:
        grad = _guarded(gradient_timing, mols[:a.grad], a, net)

    if a.profile_mode:
        a.plain_sample = 0
        a.no_cpu = True
    # ---- parity of every molecule of the timed batch against the plain FP64 path
    parity = None
    if rank == 0 and not a.profile_mode:
        parity = _guarded(batch_parity, eng, mols, a, res)
    # ---- e2e through the public batch API (b200dft.engine.run_batches): every step builds a
    # plan from the host libcint arrays of the batch's molecules (tables staged in pinned host
    # memory and copied to the device), runs the batch to convergence and copies its results to
    # host memory; the next step's plan is built on a worker thread while the GPU runs the
    # current batch.  The steps reuse the same 4096 host Mole objects (their libcint arrays are
    # built once, before timing).  The device-timed engine is released first.  This leg runs
    # before the host-heavy ones (stream workers, the CPU pool), on a quiet host.
    eng.close()
    del eng
    e2e = None
    if not a.profile_mode:
        from b200dft.engine import run_batches
        from b200dft._lib import lib as _lib
        # start from a clean device: the legs before (the float64 parity engine's 29 GB of lists)
        # leave blocks in torch's cache that the plans' own memory would otherwise have to
        # reclaim mid-run (synchronising the device)
        import gc
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        _lib().b2_release_cached_memory()
        kw = dict(level=a.level, precision=a.precision, guess=a.guess, net=net)
        for _ in run_batches([mols] * max(1, min(a.warmup, 2)), **kw):
            pass
        barrier()
        t0 = time.perf_counter()
        h2d = d2h = 0
        marks = [t0]
        host = []
        ke = max(a.steps, 10)            # at least 10 batches: one host hiccup weighs less
        import gc
        gcl = []                         # garbage-collector pauses in the timed region (ms)
        gcb = lambda ph, info: gcl.append((ph, time.perf_counter(), info.get("generation")))
        gc.callbacks.append(gcb)
        for _, out in run_batches([mols] * ke, **kw):
            host.append(dict({k: round(v, 1) for k, v in out["host_ms"].items()}, its=out["its_run"]))
            h2d += out["h2d_bytes"]
            d2h += sum(v.nbytes for v in out.values() if isinstance(v, np.ndarray))
            marks.append(time.perf_counter())
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        gc.callbacks.remove(gcb)
        gc_pauses = [round(1e3 * (b[1] - a_[1]), 1) for a_, b in zip(gcl[0::2], gcl[1::2]) if a_[2] == 2]
        barrier()
        dt = max_over_ranks(dt * 1000.0) / 1000.0
        steps_ms = [round(1e3 * (b - a_), 1) for a_, b in zip(marks[:-1], marks[1:])]
        e2e = {"value": shard.aggregate_rate(a.nmol, world, dt / ke), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d // ke), "d2h_bytes_per_step": int(d2h // ke),
               "steps": ke, "timing": "wall clock over the steps, max over ranks",
               "step_ms_min_max": [min(steps_ms), max(steps_ms)],
               "api": "b200dft.engine.run_batches (plan of the next batch prefetched on a worker thread)",
               "inputs": "the same 4096 host Mole objects (libcint arrays built before timing) every step"}
        # per-step detail goes to stderr, keeping the JSON line short
        print(json.dumps({"e2e_step_ms": steps_ms, "e2e_step_host_ms": host, "gc_gen2_pauses_ms": gc_pauses}),
              file=sys.stderr)

    learned = None
    if rank == 0 and not a.profile_mode and a.guess == "learned":
        learned = _guarded(learned_guess_criterion, mols, a, net)
    cfg2 = None
    if rank == 0 and not a.profile_mode:
        cfg2 = _guarded(config2_report)

    # ---- streaming generation (config 5): molecules generated on host workers, batched SCF with
    # slot refill and the learned guess, results to host memory, through b200dft.stream
    stream = None
    torch.cuda.empty_cache()
    if rank == 0 and not a.profile_mode and a.stream > 0:
        stream = _guarded(stream_leg, a, net, parity)

    # ---- plain FP64 per-molecule GPU path on a sample (same convergence rule, minao guess):
    # wall clock per molecule (plan, engine, eager SCF, close) and its device time
    plain = None
    if rank == 0 and a.plain_sample > 0:
        plain = _guarded(plain_leg, mols, a, res)

    # ---- CPU baseline: the reference's compiled int2e_sph + the FP64 port of its SCF on a
    # bounded sample of the batch, on a pool of the host's cores; its energies also check the
    # GPU results of the same molecules (FP64 oracle subset)
    cpu = None
    if rank == 0 and not a.no_cpu and a.cpu_sample > 0:
        cpu = _guarded(cpu_leg, a, res, parity)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": "batched uneven STO-3G B3LYP molecules (1-9 heavy atoms C/N/O/F 0.7/0.1/0.15/0.05), level-0 grid",
                       "nmol_per_gpu": a.nmol, "precision": a.precision, "guess": a.guess,
                       "l2": "inputs (s8 ERIs, grid) larger than L2 between iterations",
                       "convergence": "|dE|<1e-6 Ha and DIIS err<1e-4, retire converged"},
            "roofline": roofline, "rooflines": rooflines[1:], "parity": parity, "cpu_baseline": cpu,
            "e2e": e2e, "clocks": clocks, "gpu_launches": gpu_launches,
            "phases_ms_per_step": {k: round(v / a.steps, 3) for k, v in phase.items()},
            "scf": {"converged": int(conv.sum()), "of": int(len(conv)),
                    "fallbacks_to_minao": int(res["fell_back"].sum().item()), "mean_its": float(iters[conv].mean()) if conv.any() else None,
                    "p50_its": float(np.percentile(iters[conv], 50)) if conv.any() else None,
                    "p99_its": float(np.percentile(iters[conv], 99)) if conv.any() else None},
            "plain_fp64_per_molecule": plain, "learned_guess": learned, "config2": cfg2, "stream": stream,
        }
        if grad is not None:
            out["gradient"] = grad
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def stream_leg(a, net, parity):
    """config 5: ``a.stream`` seeded molecules of the batched distribution through
    b200dft.stream.run_stream (host generation workers, 4096 slots refilled as molecules converge,
    learned guess, rows formed on the host but not written), wall clock; plus whole batches
    without refill over the first 40960 of them, for comparison.  The plain FP64 path's
    iterations come from the whole-batch parity run (MINAO guess, same convergence rule)."""
    from b200dft.stream import run_stream
    kw = dict(batch=4096, seed=a.seed + 500, level=a.level, precision=a.precision, guess=a.guess, net=net)
    r = run_stream(a.stream, refill=True, **kw)
    nb = min(a.stream, 40960)
    rb = run_stream(nb, refill=False, **kw)
    keep = ("molecules", "wall_s", "molecules_per_s", "converged", "p50_iterations", "p99_iterations",
            "mean_iterations", "workers")
    out = {"refill": {k: r[k] for k in keep}, "whole_batches": {k: rb[k] for k in keep},
           "api": "b200dft.stream.run_stream (generation workers -> batched SCF -> host rows)"}
    if parity is not None and "plain_its" in parity:
        out["plain_fp64_iterations"] = parity["plain_its"]
    return out


def plain_leg(mols, a, res):
    """the plain FP64 per-molecule GPU path on a sample (same convergence rule, MINAO guess): wall
    clock per molecule (plan, engine, eager SCF, close) and its device time"""
    import torch
    from b200dft.engine import RKSEngine
    sample = mols[:a.plain_sample]

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plainE = []
    dev_ms = 0.0
    for m in sample:
        e1 = RKSEngine([m], level=a.level, precision="fp64")
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        r1 = e1.run_converged(graph=False)
        s1.record()
        plainE.append(float(r1["energy"][0]))
        e1.close()
        s1.synchronize()
        dev_ms += s0.elapsed_time(s1)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    dE = np.abs(np.array(plainE) - res["energy"].cpu().numpy()[:a.plain_sample])
    plain = {"value": len(sample) / dt, "unit": UNIT, "sample": len(sample),
             "device_ms_per_molecule": dev_ms / len(sample), "wall_ms_per_molecule": 1e3 * dt / len(sample),
             "max_abs_dE_batched_vs_plain_Ha": float(dE.max()),
             "timing": "wall clock over the sample (plan + engine + eager SCF + close per molecule); "
                       "device time = CUDA events around each molecule's SCF"}
    return plain


def _guarded(fn, *args):
    """an optional leg of the bench: a failure is recorded in the JSON line instead of ending the
    run (the timed value and its checks above stand on their own)"""
    try:
        return fn(*args)
    except Exception as e:  # noqa: BLE001
        import traceback
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{type(e).__name__}: {e}"}


def spawn_ranks(n):
    """``--gpus N`` without a launcher: start N ranks of this script through
    torch.distributed.run on this node (127.0.0.1) and return its exit status"""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    rc = subprocess.call(cmd)
    if rc:
        sys.exit(rc)


def _max_abs_diff_lists(x, y, plan, step=1 << 27):
    """max |x - y| over the s8 entries of every molecule of the plan (each molecule's list is
    padded to a multiple of 32 entries; the kernels never write the padding, so it is skipped)"""
    import torch
    dev = x.device
    off = torch.as_tensor(np.asarray(plan.eri_off, np.int64), device=dev)
    n2 = plan.nao.astype(np.int64) * (plan.nao.astype(np.int64) + 1) // 2
    n4 = torch.as_tensor(n2 * (n2 + 1) // 2, device=dev)
    end = int(off[-1].item() + n4[-1].item()) if len(off) else 0
    out = 0.0
    for o in range(0, end, step):
        idx = torch.arange(o, min(end, o + step), device=dev, dtype=torch.int64)
        m = torch.searchsorted(off, idx, right=True) - 1
        valid = (idx - off[m]) < n4[m]
        d = (x[o:o + idx.numel()].double() - y[o:o + idx.numel()].double()).abs()
        out = max(out, float(torch.where(valid, d, torch.zeros_like(d)).max().item()))
    return out


def batch_parity(eng, mols, a, res):
    """Every molecule of the timed batch against the plain FP64 path: the same molecules through
    the float64 engine (float64 ERIs, J/K and grid path, MINAO guess, same convergence rule;
    the float64 path matches the FP64 oracle per iteration within 1e-6 Ha in the GPU tests).
    Reports max |dE| and the count above 1e-4 Ha, max |dD| between the converged densities,
    and max |dERI| between the float32 and float64 s8 lists."""
    import torch
    from b200dft.engine import RKSEngine
    t0 = time.perf_counter()
    e64 = RKSEngine(mols, level=a.level, precision="fp64", guess="minao")   # own plan, same layout
    try:
        r64 = e64.run_converged()
        E32 = res["energy"].cpu().numpy()
        E64 = r64["energy"].cpu().numpy()
        c32 = res["converged"].cpu().numpy()
        c64 = r64["converged"].cpu().numpy()
        dE = np.abs(E32 - E64)
        dD = float((res["D"] - e64.D).abs().max().item())
        dERI = _max_abs_diff_lists(eng.eri, e64.eri, eng.plan)
        torch.cuda.synchronize()
        it64 = r64["iterations"].cpu().numpy()[c64]
        plain_its = {"p50": float(np.percentile(it64, 50)), "p99": float(np.percentile(it64, 99)),
                     "mean": float(it64.mean())} if c64.any() else None
        return {"plain_its": plain_its, "n": int(len(mols)), "reference": "plain FP64 GPU path (float64 ERIs/J/K/grid, MINAO guess), "
                                                 "same convergence rule",
                "max_abs_dE_Ha": float(dE.max()), "n_over_1e-4": int((dE > 1e-4).sum()),
                "mean_abs_dE_Ha": float(dE.mean()), "converged_mixed": int(c32.sum()), "converged_fp64": int(c64.sum()),
                "max_abs_dD": dD, "max_abs_dERI": dERI, "seconds": round(time.perf_counter() - t0, 2)}
    finally:
        e64.close()


def learned_guess_criterion(mols, a, net):
    """The learned guess's own figure: SCF iterations to DIIS error < 1e-6 (and |dE| < 1e-6 Ha)
    from the network's density vs from the MINAO-style guess, same batch, same engine."""
    from b200dft.engine import RKSEngine
    out = {"criterion": "DIIS error < 1e-6 and |dE| < 1e-6 Ha", "n": len(mols)}
    for guess in ("learned", "minao"):
        eng = RKSEngine(mols, level=a.level, precision=a.precision, guess=guess, net=net)
        try:
            r = eng.run_converged(diis_tol=1e-6, max_its=60, fallback=(guess == "learned"))
            it = r["iterations"].cpu().numpy()
            c = r["converged"].cpu().numpy()
            out[guess] = {"converged": int(c.sum()), "mean_its": float(it[c].mean()) if c.any() else None,
                          "p50_its": float(np.percentile(it[c], 50)) if c.any() else None,
                          "p99_its": float(np.percentile(it[c], 99)) if c.any() else None}
        finally:
            eng.close()
    if out["learned"]["mean_its"] and out["minao"]["mean_its"]:
        out["its_saved_per_molecule"] = out["minao"]["mean_its"] - out["learned"]["mean_its"]
    return out


def config2_report():
    """The single-molecule configuration at the size cap: the seeded 9-heavy-atom C/N/O tree on
    the level-3 grid, per precision: max |dERI| of the float32 list against the float64 list,
    max |dJ| / |dK| of the mixed J/K against the float64 J/K at the FP64 oracle's converged
    density, and |dE| of each form's 20-iteration energies against the FP64 oracle trajectory
    (committed fixture tests/golden/scf_oracle_config2_level3.npz)."""
    import torch
    from b200dft.engine import RKSEngine
    from b200dft.molgen import config2_molecule
    from b200dft.mole import Mole
    g = np.load(os.path.join(ROOT, "tests", "golden", "scf_oracle_config2_level3.npz"))
    m = Mole(config2_molecule(0))
    out = {"molecule": "config2_molecule(seed 0)", "nao": int(m.nao), "level": 3}
    engs = {}
    try:
        for prec in ("fp64", "mixed"):
            e = RKSEngine([m], level=3, precision=prec, guess="minao")
            engs[prec] = e
            t0 = time.perf_counter()
            r = e.run(its=20, log=False)
            out[prec] = {"max_abs_dE_per_iteration_Ha": float(np.abs(r["energies"][:, 0, 0] - g["energies"][:, 0]).max()),
                         "final_abs_dE_Ha": float(abs(r["energies"][-1, 0, 0] - g["energies"][-1, 0])),
                         "seconds": round(time.perf_counter() - t0, 2)}
        P = engs["fp64"].plan
        out["n_points"] = int(P.n_points)
        n4 = int(m.nao * (m.nao + 1) // 2 * (m.nao * (m.nao + 1) // 2 + 1) // 2)
        o = int(P.eri_off[0])
        out["mixed"]["max_abs_dERI"] = float((engs["mixed"].eri[o:o + n4].double() - engs["fp64"].eri[o:o + n4])
                                             .abs().max().item())
        Dref = torch.from_numpy(P.pack([g["D"]])).to(engs["fp64"].D.device)
        for e in engs.values():
            e.jk(D=Dref)
        nn = m.nao * m.nao
        out["mixed"]["max_abs_dJ"] = float((engs["mixed"].J[:nn] - engs["fp64"].J[:nn]).abs().max().item())
        out["mixed"]["max_abs_dK"] = float((engs["mixed"].K[:nn] - engs["fp64"].K[:nn]).abs().max().item())
        torch.cuda.synchronize()
    finally:
        for e in engs.values():
            e.close()
    return out


def cpu_leg(a, res, parity):
    """CPU baseline on a bounded sample of the batch (the first ``cpu_sample`` molecules): the
    reference's compiled int2e_sph (oracle/_ref) + the FP64 port of its SCF, 20 iterations, on
    spawned workers over the host's cores; the same energies check the GPU batch on those
    molecules.  Also the CH4 single-molecule time on one core (warm, second call)."""
    from oracle import eri as oeri
    from b200dft.molgen import config3_batch
    from b200dft.mole import methane
    use_ref = oeri.ref_available()
    procs = min(os.cpu_count() or 1, a.cpu_sample)
    atoms = config3_batch(a.nmol, seed=a.seed)[:a.cpu_sample]
    pool = _cpu_pool(procs, a.level, use_ref)
    try:
        v, dt, es = cpu_baseline(atoms, a.level, use_ref, pool)
    finally:
        pool.close()
        pool.join()
    Eg = res["energy"].cpu().numpy()[:len(es)]
    dE = np.abs(np.asarray(es) - Eg)
    cpu = {"value": v, "unit": UNIT, "cores": procs, "kind": "reference" if use_ref else "port",
           "sample": f"first {len(atoms)} molecules of the batch, 20 SCF iterations, FP64, {procs} worker "
                     f"processes with one BLAS thread each ({dt:.1f}s)"}
    if parity is not None:
        parity["oracle_subset"] = {"n": len(es), "max_abs_dE_Ha": float(dE.max()),
                                   "vs": "batched mixed path, converged; oracle: 20 fixed iterations"}
    cpu_baseline([methane()], a.level, use_ref)
    _, dt1, _ = cpu_baseline([methane()], a.level, use_ref)
    cpu["ch4_s_per_molecule"] = dt1
    return cpu


if __name__ == "__main__":
    main()
