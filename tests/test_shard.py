"""Multi-rank host logic on CPU (gloo, world size 2): bin partition, IQ gather,
gradient all-reduce, and the bench's per-rank step selection."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_is_disjoint_balanced_and_complete():
    from nsrno_b200.media import breast_bins
    from nsrno_b200.shard import partition_bins
    f = breast_bins()
    for world in (1, 2, 4, 8):
        parts = partition_bins(f, world)
        allb = np.concatenate(parts)
        assert sorted(allb.tolist()) == list(range(len(f)))
        loads = [f[p].sum() for p in parts]
        assert max(loads) - min(loads) <= f.max()


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from nsrno_b200.media import breast_record
        from nsrno_b200.shard import allreduce_gradient, gather_iq, shard_systems
        import bench
        rec = breast_record(nz=48, nx=64, n_pml=4, rx_pitch=1, n_rx=16)
        bins, f, a = shard_systems(rec, rank, world)
        # each rank reports its bins; gathered they cover the band exactly once
        iq = torch.tensor(np.stack([f * 1e-6 + 1j * a for _ in range(3)], axis=1), dtype=torch.complex128)
        parts = gather_iq(iq)
        grad = torch.full((2, 4, 4), float(rank + 1), dtype=torch.float64)
        allreduce_gradient(grad)
        steps = [bench.step_systems(rec, k, rank, world)[0] for k in range(3)]
        out[rank] = dict(bins=bins.tolist(), parts=[p.shape[0] for p in parts],
                         first=[complex(p[0, 0]) for p in parts], grad=float(grad[0, 0, 0]),
                         steps=[sorted(set(np.round(s).tolist())) for s in steps])
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_collectives():
    world = 2
    port = free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    b0, b1 = set(res[0]["bins"]), set(res[1]["bins"])
    assert not (b0 & b1) and len(b0 | b1) == 294
    assert res[0]["parts"] == res[1]["parts"] == [11 * len(res[0]["bins"]), 11 * len(res[1]["bins"])]
    assert res[0]["first"] == res[1]["first"]
    assert res[0]["grad"] == res[1]["grad"] == 3.0
    # bench steps: the two ranks never solve the same bin in the same step
    for k in range(3):
        assert not set(res[0]["steps"][k]) & set(res[1]["steps"][k])
