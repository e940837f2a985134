"""Replica sharding across GPUs (one process per GPU, torch.distributed).

Molecules are independent SCF problems, so N GPUs run N replicas of the batched engine on
disjoint shards of the molecule stream with no collective on the data path (the reference's
pmap over devices, nanoDFT.py:318-320, splits a batch the same way).  The only collectives are
control: a barrier around the timed region and the maximum of the per-rank elapsed times
(multi-GPU throughput = all molecules / slowest rank).
"""
import torch
import torch.distributed as dist


def shard_seed(seed, rank):
    """seed of rank ``rank``'s synthetic batch (disjoint streams per rank)"""
    return seed + 1000 * rank


def shard_indices(n_total, batch, rank, world):
    """start indices of the stream chunks of length ``batch`` owned by ``rank`` (round robin)"""
    return list(range(rank * batch, n_total, world * batch))


def max_over_ranks(x, world, device="cuda"):
    """maximum of a per-rank float over all ranks (identity when world == 1)"""
    if world == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, elapsed_s_max):
    """whole-job throughput: every rank's units over the slowest rank's time"""
    return world * units_per_rank / elapsed_s_max
