"""Replica sharding on 2 gloo ranks (CPU): disjoint shards, max-over-ranks timing, aggregate."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as tmp

from b200dft import shard
from b200dft.molgen import config3_batch, stream_molecule


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mols = config3_batch(6, seed=shard.shard_seed(11, rank), max_heavy=3)
        elapsed = 0.5 + rank                       # ranks take different times
        m = shard.max_over_ranks(elapsed, world, device="cpu")
        starts = shard.shard_indices(40, 8, rank, world)
        stream = [stream_molecule(5, i, 3) for s0 in starts for i in range(s0, min(s0 + 8, 40))]
        gathered = [None] * world
        dist.all_gather_object(gathered, {"mols": mols, "stream": stream, "max": m,
                                          "rate": shard.aggregate_rate(6, world, m)})
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    r0, r1 = res
    assert not set(r0["mols"]) & set(r1["mols"])            # disjoint synthetic shards
    assert r0["max"] == r1["max"] == 1.5                       # max over ranks on every rank
    assert r0["rate"] == r1["rate"] == pytest.approx(2 * 6 / 1.5)
    # the stream shards cover every index exactly once
    every = [stream_molecule(5, i, 3) for i in range(40)]
    assert sorted(r0["stream"] + r1["stream"]) == sorted(every)
    assert not set(r0["stream"]) & set(r1["stream"])


def test_shard_indices_round_robin():
    assert shard.shard_indices(100, 16, 0, 3) == [0, 48, 96]
    assert shard.shard_indices(100, 16, 2, 3) == [32, 80]
    assert shard.max_over_ranks(3.0, 1) == 3.0
