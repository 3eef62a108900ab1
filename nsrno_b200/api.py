"""Reference-facing entry points: drop-ins for the frequency-domain solve of NSRNO.

* :func:`solve_frequency` mirrors ``nsrno.wave_solver.solve_frequency``
  (nsrno/wave_solver.py:38-67): one medium, one frequency, one angle ->
  ``(receiver spectrum, status)``; raises ``ValueError`` on ``requires_grad`` or
  when ``max_iterations`` is not a positive multiple of ``restart``.
* :func:`solve_system` mirrors ``nsrno.dense_wave.solve_system``
  (nsrno/dense_wave.py:167-225): ``(x, info)`` with ``reason``, ``steps``,
  ``residual``, ``max_angle_residual``, ``seconds``, ``dtype``, ``method``.
* :class:`ImplicitChannels` / :func:`implicit_channels` mirror
  nsrno/dense_wave.py:227-259: a converged forward solve, receiver channels
  times the receive response, and an implicit adjoint gradient w.r.t. the
  medium ``[2, h, w] = (c, rho)``.
* :class:`HelmholtzSurrogate` mirrors ``DenseSurrogate``
  (nsrno/dense_surrogate.py:9-36): ``forward`` (differentiable) and ``truncated``.

All solves run on the GPU through ``libnsrno_b200.so``.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from . import _lib
from .solver import (DEFAULT_REPLACE, DEFAULT_SHIFT, Geometry, Medium, apply, gmres_batched, grad_accum,
                     plane_wave_rhs, receiver_response, solve_batched)

V5_CLOCK_HZ = 40e6
V5_SAMPLES = 2401


def bin_frequency(frequency_bin):
    """Frequency of a V5 record bin: ``bin * 40 MHz / 2401`` (nsrno/dense_wave.py:49)."""
    return frequency_bin * V5_CLOCK_HZ / V5_SAMPLES


class PlaneWaveModel:
    """Acquisition model for :func:`solve_frequency`: a geometry, its angles and a known alpha map.

    Stands in for the ``model`` argument of the reference (a
    ``WaveResidualOperator``), which carries the grid, the receiver columns and
    the angle table (nsrno/wave_operator.py:14-45).
    """

    def __init__(self, geometry: Geometry, angles_deg, alpha=None, warm_start=None):
        self.geometry = geometry
        self.angles = np.deg2rad(np.asarray(angles_deg, dtype=np.float64))
        self.alpha = alpha
        self.warm_start = warm_start
        self.iterations = 0 if warm_start is None else getattr(warm_start, "iterations", 1)

    def eval(self):
        return self


@torch.no_grad()
def solve_frequency(model: PlaneWaveModel, medium, frequency_hz, angle_index, tolerance=1e-4,
                    max_iterations=2560, restart=32):
    """Receiver spectrum and measured convergence status of one (frequency, angle) solve.

    ``medium`` is ``[1, 2, nz, nx]`` (c, rho).  Restarted GMRES(restart) with the
    fixed shifted-Laplace preconditioner, as nsrno/wave_solver.py:58-63.
    """
    if isinstance(medium, torch.Tensor) and medium.requires_grad:
        raise ValueError("This reference has no implicit-adjoint backward; use the neural forward for input gradients.")
    if max_iterations < restart or max_iterations % restart:
        raise ValueError("max_iterations must be a positive multiple of restart")
    started = time.perf_counter()
    g = model.geometry
    medium = torch.as_tensor(medium)
    if medium.dim() != 4 or medium.shape[0] != 1 or medium.shape[1] != 2:
        raise ValueError("One native medium per frequency solve: expected [1, 2, nz, nx]")
    dev = medium.device if medium.is_cuda else torch.device("cuda")
    alpha = model.alpha if model.alpha is not None else torch.zeros((g.nz, g.nx))
    med = Medium(g, medium[0, 0], medium[0, 1], alpha, device=dev)
    x0 = None
    if model.warm_start is not None:
        x0 = model.warm_start(med, [frequency_hz], [model.angles[angle_index]])
    res = gmres_batched(med, [frequency_hz], [model.angles[angle_index]], x0=x0, tolerance=tolerance,
                        max_iterations=max_iterations, restart=restart, n_slots=1)
    status = int(res.status[0])
    reason = "converged" if status == _lib.CONVERGED else "iteration_budget"
    iters = int(res.iterations[0])
    rel = float(res.residual[0])
    prediction = res.iq[0].to(torch.complex64)
    return prediction, dict(reason=reason, initial_neural_iterations=model.iterations,
                            solver_iterations=iters, relative_residual=rel,
                            seconds=time.perf_counter() - started,
                            trace=[dict(iterations=iters, relative_residual=rel)],
                            status=_lib.REASONS[status])


class HelmholtzSystem:
    """One medium at one frequency: the ``system`` argument of :func:`solve_system`."""

    def __init__(self, medium: Medium, frequency_hz: float):
        self.medium = medium
        self.frequency = float(frequency_hz)

    @property
    def geometry(self):
        return self.medium.geometry


@torch.no_grad()
def solve_system(system: HelmholtzSystem, rhs, preconditioner=None, adjoint=False, tolerance=1e-5,
                 max_cycles=100, warm_steps=8, mixed=False, method="gmres", initial=None,
                 max_iterations=None):
    """Solve ``A x = rhs`` (or ``A^H x = rhs``) for a batch of angles sharing one operator.

    ``rhs`` is ``[A, nz, nx]`` complex (SI units).  ``method`` is ``'gmres'``
    (restart 24, at most ``max_cycles`` cycles, nsrno/dense_wave.py:217-220),
    ``'gmres_learned'`` (the same with the learned preconditioner) or
    ``'bicgstab'``, whose unconverged angles fall back to GMRES with the fixed
    preconditioner as in nsrno/dense_wave.py:205-216.  With a
    ``preconditioner`` (:class:`~nsrno_b200.learned.LearnedPreconditioner`),
    as in nsrno/dense_wave.py:197-208: a forward solve without ``initial``
    starts from one ``warm_steps``-step GMRES cycle with the learned
    preconditioner, and BiCGSTAB uses the learned preconditioner throughout.
    The angle batch shares one frequency like the reference; every angle is
    its own Krylov system here and ``max_angle_residual`` is the largest of
    them.  ``residual`` is the combined ``||R|| / ||B||`` over all angles, as
    the reference measures it (nsrno/dense_wave.py:221-225).  ``mixed`` is
    accepted for signature compatibility: the solve always runs FP32 Krylov
    vectors against an FP64 true residual.
    """
    if method not in ("gmres", "bicgstab", "gmres_learned"):
        raise ValueError("method must be 'gmres', 'gmres_learned' or 'bicgstab'")
    started = time.perf_counter()
    med = system.medium
    g = med.geometry
    rhs = torch.as_tensor(rhs)
    squeeze = rhs.dim() == 2
    if squeeze:
        rhs = rhs[None]
    if rhs.dim() != 3 or tuple(rhs.shape[1:]) != (g.nz, g.nx):
        raise ValueError("rhs must be [A, nz, nx]")
    A = rhs.shape[0]
    b = rhs.to(med.device, torch.complex64).contiguous()
    x0 = None if initial is None else torch.as_tensor(initial).to(med.device, torch.complex64).reshape(b.shape).contiguous()
    if max_iterations is None:
        max_iterations = max_cycles * 24
    freqs = [system.frequency] * A
    setup = preconditioner.setup(med, [system.frequency]) if preconditioner is not None else None
    used_warm = 0
    if setup is not None and warm_steps and not adjoint and x0 is None:
        from .learned import warm_start
        x0, _ = warm_start(med, setup, freqs, rhs=b, steps=int(warm_steps), n_slots=A)
        used_warm = int(warm_steps)
    if method == "bicgstab":
        res = solve_batched(med, freqs, rhs=b, x0=x0, tolerance=tolerance, max_iterations=max_iterations,
                            adjoint=adjoint, return_fields=True, fields_dtype=torch.complex128, n_slots=A,
                            learned=setup)
        bad = [k for k, s in enumerate(res.status.cpu()) if int(s) != _lib.CONVERGED]
        if bad:
            # Fall back to GMRES for the angles BiCGSTAB did not converge.
            fb = gmres_batched(med, [system.frequency] * len(bad), rhs=b[bad], tolerance=tolerance,
                               max_iterations=max_cycles * 24, restart=24, adjoint=adjoint, return_fields=True,
                               fields_dtype=torch.complex128, n_slots=len(bad))
            idx = torch.as_tensor(bad, device=res.status.device)
            for name in ("residual", "status", "fields"):
                getattr(res, name)[idx] = getattr(fb, name)
            res.iterations[idx] = res.iterations[idx] * 2 + fb.iterations
    else:
        res = gmres_batched(med, freqs, rhs=b, x0=x0, tolerance=tolerance, max_iterations=max_iterations,
                            restart=24, adjoint=adjoint, return_fields=True, fields_dtype=torch.complex128,
                            n_slots=A, learned=setup if method == "gmres_learned" else None)
    bn = torch.linalg.vector_norm(rhs.reshape(A, -1).to(torch.complex128), dim=1).to(res.residual.device)
    combined = float(torch.sqrt((res.residual.square() * bn.square()).sum() / bn.square().sum().clamp_min(1e-300)))
    statuses = [int(s) for s in res.status.cpu()]
    reason = "converged" if all(s == _lib.CONVERGED for s in statuses) else _lib.REASONS[max(statuses)]
    x = res.fields.to(torch.complex128)
    if squeeze:
        x = x[0]
    steps = int(res.iterations.sum()) * (2 if method == "bicgstab" else 1) + used_warm * A
    return x, {"reason": reason, "steps": steps, "residual": combined,
               "max_angle_residual": float(res.residual.max()), "seconds": time.perf_counter() - started,
               "dtype": "complex64 Krylov / FP64 residual", "method": method,
               "iterations": [int(i) for i in res.iterations.cpu()]}


class AcquisitionData:
    """The ``data`` argument of :func:`implicit_channels`: geometry, angle table, response."""

    def __init__(self, geometry: Geometry, angles_deg, response=True):
        self.geometry = geometry
        self.angles = np.deg2rad(np.asarray(angles_deg, dtype=np.float64))
        self.response = response

    def channel_response(self, frequency_hz):
        return receiver_response(float(frequency_hz)) if self.response else 1.0


class ImplicitChannels(torch.autograd.Function):
    """Converged channels with an implicit adjoint (nsrno/dense_wave.py:227-256)."""

    @staticmethod
    def forward(ctx, medium, alpha, data, frequency_hz, angles, tolerance, max_iterations, preconditioner=None):
        g = data.geometry
        med = Medium(g, medium[0].detach(), medium[1].detach(), alpha.detach(), device=medium.device)
        th = [data.angles[a] for a in angles]
        setup = preconditioner.setup(med, [frequency_hz]) if preconditioner is not None else None
        res = solve_batched(med, [frequency_hz] * len(th), th, tolerance=tolerance, max_iterations=max_iterations,
                            return_fields=True, fields_dtype=torch.complex128, n_slots=len(th), learned=setup)
        bad = [i for i, s in enumerate(res.status.cpu()) if int(s) != _lib.CONVERGED]
        if bad:
            raise RuntimeError("Forward failed to converge: " + str({"reasons": res.reasons(),
                                                                      "residual": res.residual.tolist()}))
        resp = data.channel_response(frequency_hz)
        ctx.data, ctx.frequency, ctx.angles, ctx.tolerance, ctx.max_iterations = data, frequency_hz, th, tolerance, max_iterations
        ctx.med = med
        ctx.setup = setup
        ctx.resp = resp
        ctx.save_for_backward(medium, res.fields)
        out = res.iq * resp
        return out.to(torch.complex128)

    @staticmethod
    def backward(ctx, gradient):
        medium, u = ctx.saved_tensors
        data, med = ctx.data, ctx.med
        g = data.geometry
        A = len(ctx.angles)
        with torch.no_grad():
            rhs = torch.zeros((A, g.nz, g.nx), dtype=torch.complex64, device=medium.device)
            rx = torch.as_tensor(np.asarray(g.rx_cols), device=medium.device)
            rhs[:, g.face, rx] = (gradient * ctx.resp).to(torch.complex64)
            res = solve_batched(med, [ctx.frequency] * A, rhs=rhs, tolerance=ctx.tolerance,
                                max_iterations=ctx.max_iterations, adjoint=True, return_fields=True,
                                fields_dtype=torch.complex128, n_slots=A, learned=ctx.setup)
            bad = [i for i, s in enumerate(res.status.cpu()) if int(s) != _lib.CONVERGED]
            if bad:
                raise RuntimeError("Adjoint failed to converge: " + str({"reasons": res.reasons(),
                                                                          "residual": res.residual.tolist()}))
            g_logc, g_logrho = grad_accum(med, [ctx.frequency] * A, u, res.fields)
            grad = torch.stack((g_logc / med.c.double(), g_logrho / med.rho.double())).to(medium.dtype)
        return grad, None, None, None, None, None, None, None


def implicit_channels(medium, alpha, data, frequency_hz, angles, tolerance=1e-5, max_iterations=4000,
                      preconditioner=None):
    """Differentiable converged receiver channels ``[A, n_rx]`` (complex128).

    With a ``preconditioner`` (:class:`~nsrno_b200.learned.LearnedPreconditioner`)
    the forward and adjoint solves use the learned preconditioner (its adjoint
    for the adjoint solve), as ``ImplicitChannels`` passes its network to
    ``solve_system`` (nsrno/dense_wave.py:232-249)."""
    return ImplicitChannels.apply(medium, alpha, data, frequency_hz, list(angles), tolerance, max_iterations,
                                  preconditioner)


class HelmholtzSurrogate(torch.nn.Module):
    """Drop-in for ``DenseSurrogate`` (nsrno/dense_surrogate.py:9-36) on a synthetic record."""

    def __init__(self, geometry: Geometry, angles_deg, bins=None, response=True, device="cuda",
                 preconditioner="trained"):
        """``preconditioner``: ``"trained"`` loads the committed learned
        preconditioner (the reference surrogate loads its trained network,
        nsrno/dense_surrogate.py:11-17), ``None`` uses the fixed one, or pass a
        :class:`~nsrno_b200.learned.LearnedPreconditioner`."""
        super().__init__()
        self.data = AcquisitionData(geometry, angles_deg, response=response)
        self.bins = list(range(241, 535)) if bins is None else list(bins)
        self.device = torch.device(device)
        if isinstance(preconditioner, str):
            from .learned import LearnedPreconditioner
            preconditioner = LearnedPreconditioner.load(device=self.device)
        self.preconditioner = preconditioner

    def forward(self, medium, alpha, frequency_bin, angles=None, tolerance=1e-5):
        if frequency_bin not in self.bins:
            raise ValueError("Frequency outside cached dense band")
        angles = list(range(len(self.data.angles))) if angles is None else list(angles)
        return implicit_channels(medium, alpha, self.data, bin_frequency(frequency_bin), angles, tolerance,
                                 preconditioner=self.preconditioner)

    @torch.no_grad()
    def truncated(self, medium, alpha, frequency_bin, angles=None, iterations=32):
        """Channels after one GMRES cycle of ``iterations`` Arnoldi steps with the
        learned preconditioner, and the actual relative residual of that field
        over all requested angles (``DenseSurrogate.truncated``,
        nsrno/dense_surrogate.py:30-36, through ``batched_gmres_cycle``,
        nsrno/dense_wave.py:84-116).  Each angle has its own Krylov space here
        (the reference shares one across the angles of a bin); the per-angle
        minimisation can only lower the joint residual the reference reports.
        More than 64 steps run as cycles of 64."""
        if frequency_bin not in self.bins:
            raise ValueError("Frequency outside cached dense band")
        if iterations < 1:
            raise ValueError("iterations must be >= 1")
        angles = list(range(len(self.data.angles))) if angles is None else list(angles)
        g = self.data.geometry
        med = Medium(g, medium[0], medium[1], alpha, device=medium.device)
        f = bin_frequency(frequency_bin)
        th = [self.data.angles[a] for a in angles]
        setup = self.preconditioner.setup(med, [f]) if self.preconditioner is not None else None
        restart = min(int(iterations), 64)
        res = gmres_batched(med, [f] * len(th), th, tolerance=1e-30, max_iterations=int(iterations), restart=restart,
                            n_slots=len(th), learned=setup)
        b = plane_wave_rhs(med, [f] * len(th), th)
        bn = b.flatten(1).norm(dim=1)
        joint = float(torch.sqrt(((res.residual * bn) ** 2).sum() / (bn ** 2).sum()))
        resp = self.data.channel_response(f)
        return (res.iq * resp).to(torch.complex128), joint
