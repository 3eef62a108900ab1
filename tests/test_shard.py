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


class _LinearGN:
    """A Gauss-Newton step on a linear model r = J m - d, split by rows over ranks."""

    @staticmethod
    def make(rank, world, distributed):
        from nsrno_b200.gauss_newton import GaussNewton

        class Fake(GaussNewton):
            def __post_init__(self):
                rng = np.random.default_rng(7)
                self.J = torch.as_tensor(rng.standard_normal((24, 2 * 9)))     # 24 receivers, 2 planes of 3x3
                self.d = torch.as_tensor(rng.standard_normal(24))
                rows = np.array_split(np.arange(24), world)[rank] if distributed else np.arange(24)
                self.J, self.d = self.J[rows], self.d[rows]

            def forward(self):
                self.r = -self.d
                return 0.5 * float((self.r ** 2).sum())

            def gradient(self):
                g = self.J.T @ self.r
                return g[:9].reshape(3, 3), g[9:].reshape(3, 3)

            def hessian_vector(self, vc, vr):
                jv = self.J @ torch.cat((vc.reshape(-1), vr.reshape(-1)))
                h = self.J.T @ jv
                return (h[:9].reshape(3, 3), h[9:].reshape(3, 3)), jv

        return Fake(medium=None, freqs=np.zeros(1), angles=np.zeros(1), d_obs=None, distributed=distributed)


def _gn_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        step = _LinearGN.make(rank, world, True).step()
        out[rank] = dict(alpha=step["alpha"], misfit=step["misfit"], vhv=step["vHv"], jv2=step["jv_norm2"],
                         update=step["update"][0].numpy().tolist())
    finally:
        dist.destroy_process_group()


def test_gauss_newton_step_sums_over_ranks():
    """Two gloo ranks holding halves of the systems take the same step as one
    process holding all of them: misfit, gradient and H v are all-reduced."""
    whole = _LinearGN.make(0, 1, False).step()
    world, port = 2, free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_gn_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        assert res[r]["alpha"] == pytest.approx(whole["alpha"], rel=1e-12)
        assert res[r]["misfit"] == pytest.approx(whole["misfit"], rel=1e-12)
        assert res[r]["vhv"] == pytest.approx(whole["vHv"], rel=1e-12)
        assert res[r]["jv2"] == pytest.approx(whole["jv_norm2"], rel=1e-12)
        assert np.allclose(res[r]["update"], whole["update"][0].numpy(), rtol=1e-12)
