"""Sharding of a record's systems over GPUs (one process per GPU).

The (frequency, angle) systems of a record are independent, so the forward
solve needs no collective: each rank solves whole frequency bins (all angles of
a bin on one rank, so they share the coefficient planes and the preconditioner
symbol).  Two exchanges exist around it, as in the reference's DDP drivers
(nsrno/reconstruct_dense.py:53,97-118): gathering receiver IQ once per record
and summing the material gradient of an inversion step.
"""
from __future__ import annotations

import heapq

import numpy as np
import torch
import torch.distributed as dist


def partition_bins(frequencies, world, cost=None):
    """Longest-first greedy assignment of bins to ranks.

    Iteration counts grow with frequency, so the default cost of a bin is its
    frequency.  Returns one sorted array of bin indices per rank.
    """
    frequencies = np.asarray(frequencies, dtype=np.float64)
    cost = frequencies if cost is None else np.asarray(cost, dtype=np.float64)
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for b in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(b))
        heapq.heappush(heap, (load + float(cost[b]), r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def shard_systems(record, rank, world):
    """(bins, freqs, angles) of this rank: every angle of its bins, highest frequency first."""
    bins = partition_bins(record.frequencies, world)[rank]
    bins = bins[np.argsort(-record.frequencies[bins], kind="stable")]
    f = np.repeat(record.frequencies[bins], len(record.angles))
    a = np.tile(record.angles, len(bins))
    return bins, f, a


def gather_iq(iq: torch.Tensor, group=None):
    """All-gather per-rank receiver IQ ``[S_rank, n_rx]`` (complex) into a list by rank."""
    world = dist.get_world_size(group)
    real = torch.view_as_real(iq.contiguous())
    count = torch.tensor([real.shape[0]], dtype=torch.int64, device=real.device)
    counts = [torch.zeros_like(count) for _ in range(world)]
    dist.all_gather(counts, count, group=group)
    top = int(max(int(c) for c in counts))
    padded = torch.zeros((top,) + tuple(real.shape[1:]), dtype=real.dtype, device=real.device)
    padded[: real.shape[0]] = real
    bufs = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(bufs, padded, group=group)
    return [torch.view_as_complex(b[: int(c)].contiguous()) for b, c in zip(bufs, counts)]


def allreduce_gradient(grad: torch.Tensor, group=None):
    """Sum the material gradient ``[2, nz, nx]`` over ranks in place (one all-reduce)."""
    dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad
