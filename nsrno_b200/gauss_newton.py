"""Gauss-Newton step of the frequency-domain inversion on one GPU.

One step over a record's (frequency, angle) systems:

* forward solves ``A u = s`` (learned preconditioner), receiver residual
  ``r = P u - d_obs`` and misfit ``0.5 |r|^2``;
* adjoint solves ``A^H lam = P^T r`` and the gradient
  ``g = -Re(lam^H dA/dm u)`` for m = (log c, log rho) (``nsr_grad_accum``);
* for a direction v: tangent solves ``A du = -dA[v] u`` (``nsr_tangent_rhs``,
  the Born perturbation of theranostic/wave.py:280-329), ``J v = P du``, a
  second adjoint solve ``A^H mu = P^T J v`` and the Gauss-Newton
  Hessian-vector product ``H v = Re(J^H J v) = -Re(mu^H dA/dm u)``;
* the exact Gauss-Newton step length along v, ``alpha = -<g, v>/<v, H v>``.

The reference's only tangent is time-domain (nsrno/native_tangent.cu:53-79);
the frequency-domain one reuses the batched solver with a tangent right-hand
side.  All fields of a step stay resident on the device (c64 background and
adjoint fields: 8 bytes per node and system).

On several GPUs (one process per GPU, ``distributed=True``) every rank holds
the systems of its own frequency bins; the misfit, the gradient and the
Hessian-vector product are sums over systems, so each is one all-reduce
(the gradient all-reduce of the reference's DDP inversion,
nsrno/reconstruct_dense.py:53,97-106), and every rank then takes the same step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .solver import Geometry, Medium, _ptr, _require_cuda, _stream, grad_accum, solve_batched


def tangent_rhs(medium: Medium, freqs, u: torch.Tensor, dlogc, dlogrho):
    """``-dA[dm] u`` in SI units for background fields u [S, nz, nx] (c64 or c128)."""
    g = medium.geometry
    _require_cuda(u, "u")
    if u.dtype not in (torch.complex64, torch.complex128) or u.dim() != 3 or tuple(u.shape[1:]) != (g.nz, g.nx):
        raise ValueError("u must be complex64/complex128 [S, nz, nx]")
    u = u.contiguous()
    dev = u.device
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    if freqs.numel() != u.shape[0]:
        raise ValueError("one frequency per field")
    dc = torch.as_tensor(dlogc, dtype=torch.float64, device=dev).reshape(g.nz, g.nx).contiguous()
    dr = torch.as_tensor(dlogrho, dtype=torch.float64, device=dev).reshape(g.nz, g.nx).contiguous()
    out = torch.empty_like(u)
    _lib.check(_lib.load().nsr_tangent_rhs(ctypes.byref(medium._grid), _ptr(medium.material), _ptr(freqs), u.shape[0],
                                           int(u.dtype == torch.complex128), _ptr(u), _ptr(dc), _ptr(dr), _ptr(out),
                                           _stream()))
    return out


def _require_converged(res, what, tolerance=None, accept_factor=1.0):
    """Raise unless every system converged.  With ``accept_factor`` > 1, a
    system that used its whole iteration budget but whose FP64 true residual
    is within ``accept_factor * tolerance`` is accepted; returns how many."""
    status = res.status.cpu()
    resid = res.residual.cpu()
    near = [i for i, s in enumerate(status) if int(s) == _lib.ITERATION_BUDGET and tolerance is not None
            and float(resid[i]) <= accept_factor * tolerance]
    bad = [i for i, s in enumerate(status) if int(s) != _lib.CONVERGED and i not in set(near)]
    if bad:
        raise RuntimeError(f"{what} failed to converge for {len(bad)} systems: "
                           f"{sorted(set(res.reasons()))}, max residual {float(res.residual.max()):.3g}")
    return len(near)


@dataclass
class GaussNewton:
    """A record's systems, observed receiver data and the solver settings of one step."""

    medium: Medium
    freqs: np.ndarray                 # [S]
    angles: np.ndarray                # [S]
    d_obs: torch.Tensor               # complex128 [S, n_rx]
    preconditioner: object = None     # LearnedPreconditioner or None (fixed shifted Laplace)
    tolerance: float = 1e-6
    n_slots: int = 22
    max_iterations: int = 2000
    # Adjoint solves with receiver-row sources can stall just above the
    # tolerance at the accuracy the FP32 operator allows (a few of the
    # band's highest frequencies at 0.04 mm): such a system is accepted when
    # its FP64 true residual is within this factor of the tolerance, and
    # counted in `near_tolerance`.
    accept_factor: float = 2.0
    distributed: bool = False         # sum misfit, gradient and H v over the ranks of `group`
    group: object = None              # torch.distributed process group (None: the default group)
    timings: dict = field(default_factory=dict)
    near_tolerance: dict = field(default_factory=dict)   # per solve kind: systems accepted within accept_factor

    def __post_init__(self):
        dev = self.medium.device
        self.freqs = np.asarray(self.freqs, dtype=np.float64)
        self.angles = np.asarray(self.angles, dtype=np.float64)
        self.f_dev = torch.as_tensor(self.freqs, device=dev)
        self.setup = None
        if self.preconditioner is not None:
            self.setup = self.preconditioner.setup(self.medium, torch.unique(self.f_dev))
        self.u = None

    def _solve(self, what, fields=True, **kw):
        t0 = time.perf_counter()
        res = solve_batched(self.medium, self.f_dev, tolerance=self.tolerance, max_iterations=self.max_iterations,
                            n_slots=self.n_slots, learned=self.setup, return_fields=fields, **kw)
        torch.cuda.synchronize()
        self.timings[what] = self.timings.get(what, 0.0) + time.perf_counter() - t0
        self.near_tolerance[what] = _require_converged(res, what, self.tolerance, self.accept_factor)
        return res

    def _receiver_rhs(self, values):
        g = self.medium.geometry
        S = len(self.freqs)
        rhs = torch.zeros((S, g.nz, g.nx), dtype=torch.complex64, device=self.medium.device)
        rx = torch.as_tensor(np.asarray(g.rx_cols), device=self.medium.device)
        rhs[:, g.face, rx] = values.to(torch.complex64)
        return rhs

    def forward(self):
        res = self._solve("forward", angles=torch.as_tensor(self.angles, device=self.medium.device))
        self.u = res.fields
        self.iq = res.iq
        self.r = res.iq - self.d_obs
        self.forward_result = res
        return 0.5 * float((self.r.abs() ** 2).sum())

    def gradient(self):
        """``(g_logc, g_logrho)`` of the misfit, float64 [nz, nx] each."""
        lam = self._solve("adjoint", rhs=self._receiver_rhs(self.r), adjoint=True).fields
        t0 = time.perf_counter()
        g = grad_accum(self.medium, self.f_dev, self.u, lam)
        torch.cuda.synchronize()
        self.timings["gradient"] = self.timings.get("gradient", 0.0) + time.perf_counter() - t0
        return g

    def jvp(self, dlogc, dlogrho):
        """``J v``: receiver perturbation [S, n_rx] of the direction v = (dlogc, dlogrho)."""
        t0 = time.perf_counter()
        rhs = tangent_rhs(self.medium, self.f_dev, self.u, dlogc, dlogrho)
        self.timings["tangent_rhs"] = self.timings.get("tangent_rhs", 0.0) + time.perf_counter() - t0
        iq = self._solve("tangent", fields=False, rhs=rhs).iq
        del rhs
        return iq

    def hessian_vector(self, dlogc, dlogrho):
        """``(H v, J v)`` of the Gauss-Newton Hessian ``Re(J^H J)``."""
        jv = self.jvp(dlogc, dlogrho)
        mu = self._solve("adjoint2", rhs=self._receiver_rhs(jv), adjoint=True).fields
        return grad_accum(self.medium, self.f_dev, self.u, mu), jv

    def _sum_planes(self, a, b):
        """(a, b) summed over the ranks: one all-reduce of the stacked planes."""
        if not self.distributed:
            return a, b
        from .shard import allreduce_gradient
        t0 = time.perf_counter()
        both = allreduce_gradient(torch.stack((a, b)).contiguous(), group=self.group)
        self.timings["allreduce"] = self.timings.get("allreduce", 0.0) + time.perf_counter() - t0
        return both[0], both[1]

    def _sum_scalar(self, x, like):
        if not self.distributed:
            return float(x)
        import torch.distributed as dist
        t = torch.tensor([float(x)], dtype=torch.float64, device=like.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return float(t)

    def step(self):
        """One step along the steepest-descent direction with the exact Gauss-Newton length."""
        self.timings = {}
        t0 = time.perf_counter()
        misfit = self.forward()
        gc, gr = self._sum_planes(*self.gradient())
        misfit = self._sum_scalar(misfit, gc)
        gnorm = float(torch.sqrt((gc ** 2).sum() + (gr ** 2).sum()))
        vc, vr = -gc / gnorm, -gr / gnorm
        (hc, hr), jv = self.hessian_vector(vc, vr)
        hc, hr = self._sum_planes(hc, hr)
        gv = float((gc * vc).sum() + (gr * vr).sum())
        vhv = float((vc * hc).sum() + (vr * hr).sum())
        alpha = -gv / vhv
        jv2 = self._sum_scalar((jv.abs() ** 2).sum(), gc)
        total = time.perf_counter() - t0
        return dict(misfit=misfit, gradient_norm=gnorm, vHv=vhv, jv_norm2=jv2,
                    alpha=alpha, predicted_decrease=0.5 * gv * gv / vhv, seconds=total,
                    phase_seconds=dict(self.timings), near_tolerance=dict(self.near_tolerance),
                    update=(alpha * vc, alpha * vr))


def main():
    """Time one Gauss-Newton step on a synthetic breast record (default: 1536 x 1024 nodes at 0.04 mm,
    11 angles x the 294 bins; ``--bins`` takes a subset spread over the band)."""
    from .learned import LearnedPreconditioner
    from .media import breast_bins, breast_record, perturbed
    ap = argparse.ArgumentParser()
    ap.add_argument("--nz", type=int, default=1024)
    ap.add_argument("--nx", type=int, default=1536)
    ap.add_argument("--h", type=float, default=4e-5)
    ap.add_argument("--bins", type=int, default=294)
    ap.add_argument("--angles", type=int, default=11)
    ap.add_argument("--slots", type=int, default=22)
    ap.add_argument("--fixed", action="store_true", help="fixed shifted-Laplace preconditioner")
    a = ap.parse_args()
    import os
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        # one process per GPU (torchrun); each rank solves its own bins
        import datetime
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda")
    all_bins = breast_bins()
    pick = np.unique(np.linspace(0, len(all_bins) - 1, a.bins).round().astype(int))
    if world > 1:
        from .shard import partition_bins
        pick = pick[partition_bins(all_bins[pick], world)[rank]]
    rec = breast_record(nz=a.nz, nx=a.nx, h=a.h, n_pml=int(round(1.2e-3 / a.h)), bins=all_bins[pick],
                        n_angles=a.angles, rx_pitch=max(1, int(round(2e-4 / a.h))))
    true = perturbed(rec, seed=3)
    f, th = rec.systems()
    geo = Geometry.from_record(rec)
    pre = None if a.fixed else LearnedPreconditioner.load(device=dev)
    t0 = time.perf_counter()
    m_true = Medium(geo, true.c, true.rho, true.alpha, device=dev)
    setup = pre.setup(m_true, torch.unique(torch.as_tensor(f, device=dev))) if pre is not None else None
    obs = solve_batched(m_true, f, th, tolerance=1e-6, max_iterations=6000, n_slots=a.slots, learned=setup)
    _require_converged(obs, "observed data")
    del setup
    t_obs = time.perf_counter() - t0
    med = Medium(geo, rec.c, rec.rho, rec.alpha, device=dev)
    gn = GaussNewton(med, f, th, obs.iq, preconditioner=pre, n_slots=a.slots, distributed=world > 1)
    torch.cuda.reset_peak_memory_stats()
    out = gn.step()
    out.pop("update")
    fw = gn.forward_result
    # FP64 spot checks: 8 systems spread over the band re-solved to a 1e-10 FP64
    # true residual; the receiver IQ of the 1e-6 forward solves against them.
    spot = np.unique(np.linspace(0, len(f) - 1, 8).round().astype(int))
    ref = solve_batched(med, f[spot], th[spot], tolerance=1e-10, max_iterations=20000, n_slots=len(spot),
                        learned=gn.setup)
    _require_converged(ref, "FP64 spot check")
    diff = (fw.iq[torch.as_tensor(spot, device=dev)] - ref.iq).norm(dim=1) / ref.iq.norm(dim=1)
    out.update(spot_systems=spot.tolist(), spot_iq_rel_error_max=float(diff.max()),
               spot_iq_rel_error_mean=float(diff.mean()), spot_residual_max=float(ref.residual.max()))
    out.update(grid_zx=[a.nz, a.nx], h=a.h, systems=len(f), bins=len(pick), angles=a.angles,
               preconditioner="fixed" if a.fixed else "learned", observed_data_seconds=t_obs,
               solves_per_step=4 * len(f), solves_per_second=4 * len(f) / out["seconds"],
               forward_iterations_mean=float(fw.iterations.float().mean()),
               forward_residual_max=float(fw.residual.max()),
               peak_device_gb=torch.cuda.max_memory_allocated() / 1e9, ranks=world)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
