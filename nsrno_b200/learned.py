"""Learned preconditioner of the 5-point path: set-up, apply, warm start and training.

The network is the reference's ``LearnedPreconditioner``
(nsrno/conditioned_wave.py:94-117) with its 3,645 parameters in the order of
that module's ``state_dict``; ``learned_apply`` (nsrno/dense_wave.py:150-165)
and the 8-step GMRES warm start of ``solve_system`` (dense_wave.py:197-201) use
it the same way here.  On the 5-point grid the map is the complex conjugate of
the reference's (this path's ``exp(-i omega t)`` convention) in the units of
the h^2-scaled operator; with an untrained network it is exactly the fixed
shifted-Laplace preconditioner.

Training (:func:`train`) runs on the GPU through this library's kernels:
``nsr_learned_setup`` (network forward), ``nsr_learned_precondition`` and
``nsr_apply`` (the minimal-residual iterations), and the backward kernels
``nsr_learned_map_backward``, ``nsr_learned_network_backward`` and
``nsr_learned_spectral_backward``, then ``nsr_learned_adam``.  The objective
follows the reference's training model (nsrno/train_dense_wave.py:14-21,66-68:
a relative receiver error plus the relative PDE residual of a truncated
Krylov solve with the learned preconditioner), in log form, with the
receiver targets taken from this solver's own converged solves.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .solver import Geometry, Medium, _ptr, _require_cuda, _stream, apply, plane_wave_rhs, solve_batched

N_PARAMS = _lib.LEARNED_PARAMS
SHAPES = (("spectral", (2, 4)), ("log_shift", ()), ("context.0.weight", (16, 5, 3, 3)), ("context.0.bias", (16,)),
          ("context.2.weight", (16, 16, 3, 3)), ("context.2.bias", (16,)), ("context.4.weight", (4, 16, 3, 3)),
          ("context.4.bias", (4,)))
WEIGHTS = Path(__file__).resolve().parent / "weights" / "learned_5pt.npz"


def initial_parameters(seed=0):
    """Untrained parameters (conditioned_wave.py:96-101): PyTorch's default
    uniform initialisation of the first two convolutions, a zero last layer,
    zero spectral weights and ``log(0.15)`` -- identity gains."""
    g = torch.Generator().manual_seed(seed)
    parts = []
    for name, shape in SHAPES:
        size = int(np.prod(shape)) if shape else 1
        if name in ("context.0.weight", "context.2.weight", "context.0.bias", "context.2.bias"):
            fan_in = (5 if name.startswith("context.0") else 16) * 9
            parts.append((torch.rand(size, generator=g, dtype=torch.float64) * 2 - 1) / math.sqrt(fan_in))
        elif name == "log_shift":
            parts.append(torch.tensor([math.log(0.15)], dtype=torch.float64))
        else:
            parts.append(torch.zeros(size, dtype=torch.float64))
    return torch.cat(parts).to(torch.float32)


@dataclass
class LearnedSetup:
    """Gains of one medium at a list of frequencies, ready for the solvers."""

    params: torch.Tensor      # float32 [3645] (device)
    freqs: torch.Tensor       # float64 [F] (device)
    state: torch.Tensor       # network activations (device bytes)
    gains: torch.Tensor       # complex64 [F, 2, nz, nx]: inner, outer
    precision: int = 0        # _lib.LEARNED_FP32 or LEARNED_BF16 (the state's planes)

    @property
    def n_gain(self):
        return int(self.freqs.numel())

    def struct(self, gain_index=None):
        return _lib.NsrLearned(self.params.data_ptr(), self.gains.data_ptr(),
                               0 if gain_index is None else gain_index.data_ptr(), self.n_gain, 0)

    def index_of(self, freqs):
        """Gain pair of each system: the set-up frequency equal to its frequency."""
        f = torch.as_tensor(freqs, dtype=torch.float64, device=self.freqs.device).reshape(-1)
        d = (f[:, None] - self.freqs[None, :]).abs()
        idx = d.argmin(dim=1)
        if bool((d.gather(1, idx[:, None]).squeeze(1) > 1e-6 * f.abs().clamp_min(1.0)).any()):
            raise ValueError("a system frequency has no learned gains; set up every frequency first")
        return idx.to(torch.int32)


class LearnedPreconditioner:
    """Parameters of the learned preconditioner on one device."""

    def __init__(self, params=None, device=None, precision="fp32"):
        """``precision``: ``"fp32"`` or ``"bf16"`` -- the network's weights and
        activations in bfloat16 with every product accumulated in FP32 (the
        parameters themselves, their gradients and Adam stay FP32)."""
        device = torch.device(device or "cuda")
        p = initial_parameters() if params is None else torch.as_tensor(params, dtype=torch.float32).reshape(-1)
        if p.numel() != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters, got {p.numel()}")
        if precision not in _lib.PRECISIONS:
            raise ValueError("precision must be 'fp32' or 'bf16'")
        self.params = p.to(device).contiguous()
        self.precision = precision
        self.meta = {}

    @classmethod
    def load(cls, path=WEIGHTS, device=None, precision=None):
        """Committed weights; ``precision`` defaults to the one they were trained in."""
        with np.load(path) as z:
            meta = json.loads(str(z["meta"])) if "meta" in z.files else {}
            obj = cls(z["params"], device=device, precision=precision or meta.get("precision", "fp32"))
            obj.meta = meta
        return obj

    def save(self, path, **meta):
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, params=self.params.detach().cpu().numpy(), meta=json.dumps({**self.meta, **meta}))

    @property
    def device(self):
        return self.params.device

    @property
    def shift(self):
        return float(min(max(math.exp(float(self.params[8])), 0.01), 1.0))

    def setup(self, medium: Medium, freqs) -> LearnedSetup:
        """Network forward and gains of ``medium`` at every frequency in ``freqs``."""
        g = medium.geometry
        lib = _lib.load()
        freqs = torch.as_tensor(freqs, dtype=torch.float64, device=medium.device).reshape(-1).contiguous()
        F = int(freqs.numel())
        nbytes = lib.nsr_learned_state_bytes(ctypes.byref(medium._grid), max(F, 1))
        if nbytes == 0:
            raise ValueError("unsupported grid for the learned preconditioner")
        state = torch.empty(nbytes, dtype=torch.uint8, device=medium.device)
        gains = torch.empty((F, 2, g.nz, g.nx), dtype=torch.complex64, device=medium.device)
        prec = _lib.PRECISIONS[getattr(self, "precision", "fp32")]
        _lib.check(lib.nsr_learned_setup_ex(ctypes.byref(medium._grid), _ptr(medium.c), _ptr(medium.rho),
                                            _ptr(medium.alpha), _ptr(freqs), F, _ptr(self.params), prec,
                                            _ptr(state), _ptr(gains), _stream()))
        return LearnedSetup(self.params, freqs, state, gains, prec)


def learned_precondition(medium: Medium, setup: LearnedSetup | None, x: torch.Tensor, freqs, adjoint=False,
                         gain_index=None, params=None):
    """``M x`` (or ``M^H x``) of the learned preconditioner for complex64 fields [S, nz, nx].

    With ``setup=None`` only the learned spectral multiplier of ``params`` is
    applied (no diagonal gains)."""
    g = medium.geometry
    _require_cuda(x, "x")
    if x.dtype != torch.complex64 or x.dim() != 3 or tuple(x.shape[1:]) != (g.nz, g.nx):
        raise ValueError("x must be complex64 [S, nz, nx]")
    x = x.contiguous()
    S = x.shape[0]
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=x.device).reshape(-1).contiguous()
    lib = _lib.load()
    nbytes = lib.nsr_precondition_workspace_size(ctypes.byref(medium._grid), S)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
    y = torch.empty_like(x)
    if setup is not None:
        if gain_index is None:
            gain_index = setup.index_of(freqs)
        gain_index = torch.as_tensor(gain_index, dtype=torch.int32, device=x.device).contiguous()
        struct = setup.struct(gain_index)
    else:
        struct = _lib.NsrLearned(params.data_ptr(), 0, 0, 0, 0)
    _lib.check(lib.nsr_learned_precondition(ctypes.byref(medium._grid), ctypes.byref(struct), _ptr(freqs), S,
                                            int(bool(adjoint)), _ptr(x), _ptr(y), _ptr(ws), nbytes, _stream()))
    return y


def warm_start(medium: Medium, setup: LearnedSetup, freqs, angles=None, *, rhs=None, steps=8, adjoint=False,
               gain_index=None, n_slots=16):
    """Initial fields from one GMRES cycle of ``steps`` Arnoldi steps with the
    learned preconditioner (``batched_gmres_cycle`` with the learned setup,
    nsrno/dense_wave.py:84-116,197-201); complex64 [S, nz, nx]."""
    from .solver import gmres_batched
    res = gmres_batched(medium, freqs, angles, rhs=rhs, tolerance=1e-30, max_iterations=steps, restart=steps,
                        n_slots=n_slots, adjoint=adjoint, return_fields=True, learned=setup, gain_index=gain_index)
    return res.fields, res


# ---------------------------------------------------------------------------
# Training
# ---------------------------------------------------------------------------
def _dot(a, b):
    """Per-system <a, b> = sum conj(a) b, complex128 [S]."""
    return (a.conj() * b).flatten(1).to(torch.complex128).sum(dim=1)


def _bc(v):
    return v.to(torch.complex64)[:, None, None]


@dataclass
class Batch:
    """One training batch: a medium and S (frequency, angle) systems with receiver targets."""

    medium: Medium
    freqs: torch.Tensor       # float64 [S]
    angles: torch.Tensor      # float64 [S]
    rhs: torch.Tensor         # complex64 [S, nz, nx], h^2 units
    rx: torch.Tensor          # int64 [n_rx] flat receiver nodes
    target: torch.Tensor | None   # complex128 [S, n_rx]: converged receiver IQ


def make_batch(medium: Medium, freqs, angles, with_target=True, tolerance=1e-6):
    g = medium.geometry
    dev = medium.device
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1)
    angles = torch.as_tensor(angles, dtype=torch.float64, device=dev).reshape(-1)
    rhs = (plane_wave_rhs(medium, freqs, angles) * g.h ** 2).to(torch.complex64)
    rx = g.rx_index(dev).long()
    target = None
    if with_target:
        res = solve_batched(medium, freqs, angles, tolerance=tolerance, max_iterations=6000,
                            n_slots=int(freqs.numel()))
        bad = [k for k, s in enumerate(res.status.cpu()) if int(s) != _lib.CONVERGED]
        if bad:
            # GMRES for the systems BiCGSTAB did not converge (the fallback of solve_system)
            from .solver import gmres_batched
            idx = torch.as_tensor(bad, device=dev)
            fb = gmres_batched(medium, freqs[idx], angles[idx], tolerance=tolerance, max_iterations=20000,
                               restart=32, n_slots=len(bad))
            if fb.reasons() != ["converged"] * len(bad):
                raise RuntimeError(f"target solve did not converge: {fb.reasons()}")
            res.iq[idx] = fb.iq
        target = res.iq
    return Batch(medium, freqs, angles, rhs, rx, target)


def loss_and_grad(params: torch.Tensor, batch: Batch, steps: int, channel_weight=1.0, precision="fp32"):
    """Loss and exact gradient w.r.t. all parameters (hand-written backward kernels).

    Loss (mean over the batch's systems) after ``steps`` minimal-residual
    iterations from zero with the learned preconditioner M:

        z = M r,  w = A z,  g = <w, r>/<w, w>,  x += g z,  r -= g w,
        L = log(|r|^2/|b|^2) + channel_weight * log(|x[rx] - d|^2/|d|^2).
    """
    lib = _lib.load()
    med = batch.medium
    grid = ctypes.byref(med._grid)
    S = int(batch.freqs.numel())
    pre = LearnedPreconditioner.__new__(LearnedPreconditioner)
    pre.params = params
    pre.precision = precision
    setup = pre.setup(med, batch.freqs)
    inner, outer = setup.gains[:, 0], setup.gains[:, 1]
    core = lambda v, adj=False: learned_precondition(med, None, v, batch.freqs, adjoint=adj, params=params)
    b = batch.rhs
    r = b.clone()
    x = torch.zeros_like(b)
    saved = []
    for _ in range(steps):
        q = core(inner * r)
        z = outer * q
        w = apply(med, z, batch.freqs)
        ww = _dot(w, w).real
        gam = _dot(w, r) / ww
        saved.append((r, q, z, w, gam, ww))
        x = x + _bc(gam) * z
        r = r - _bc(gam) * w
    bb = _dot(b, b).real
    rr = _dot(r, r).real
    loss_sys = torch.log(rr / bb)
    Rbar = r * (1.0 / rr).to(torch.float32)[:, None, None] / S
    Xbar = torch.zeros_like(x)
    if batch.target is not None and channel_weight:
        d = x.flatten(1)[:, batch.rx].to(torch.complex128)
        e = d - batch.target
        ee = (e.abs() ** 2).sum(dim=1)
        tt = (batch.target.abs() ** 2).sum(dim=1)
        loss_sys = loss_sys + channel_weight * torch.log(ee / tt)
        Xbar.view(S, -1)[:, batch.rx] = (channel_weight * e / ee[:, None] / S).to(torch.complex64)
    g_in = torch.zeros_like(b)
    g_out = torch.zeros_like(b)
    grad = torch.zeros(N_PARAMS, dtype=torch.float32, device=params.device)
    spec_bytes = lib.nsr_learned_spectral_workspace_size(grid, S)
    if spec_bytes == 0:
        raise ValueError("grid too large for the spectral backward kernel")
    spec_ws = torch.empty(spec_bytes, dtype=torch.uint8, device=params.device)
    for (rk, qk, zk, wk, gam, ww) in reversed(saved):
        ct = _dot(Rbar, wk) - _dot(Xbar, zk)
        Wbar = (-_bc(gam.conj()) * Rbar - _bc(ct / ww) * rk + _bc(2.0 * (ct * gam).real / ww) * wk)
        Rprev = Rbar - _bc(ct.conj() / ww) * wk
        Zbar = apply(med, Wbar, batch.freqs, adjoint=True) + _bc(gam.conj()) * Xbar
        g_out += Zbar * qk.conj()
        Y = outer.conj() * Zbar
        Ybar = core(Y, adj=True)
        u = inner * rk
        g_in += Ybar * rk.conj()
        _lib.check(lib.nsr_learned_spectral_backward(grid, _ptr(params), _ptr(batch.freqs), S, _ptr(u), _ptr(Y),
                                                     _ptr(grad), _ptr(spec_ws), spec_bytes, _stream()))
        Rbar = Rprev + inner.conj() * Ybar
    bw_bytes = lib.nsr_learned_backward_workspace_size(grid, S)
    bw = torch.empty(bw_bytes, dtype=torch.uint8, device=params.device)
    g = med.geometry
    d_maps = torch.empty((S, 4, g.nz // 8, g.nx // 8), dtype=torch.float32, device=params.device)
    _lib.check(lib.nsr_learned_map_backward_ex(grid, _ptr(setup.state), setup.precision, S, _ptr(g_in.contiguous()),
                                               _ptr(g_out.contiguous()), _ptr(d_maps), _ptr(bw), bw_bytes,
                                               _stream()))
    _lib.check(lib.nsr_learned_network_backward_ex(grid, _ptr(params), _ptr(setup.state), setup.precision, S,
                                                   _ptr(d_maps), _ptr(grad), _ptr(bw), bw_bytes, _stream()))
    return float(loss_sys.mean()), grad, [float(v) for v in loss_sys]


class Adam:
    """Adam with gradient-norm clipping on the device (``nsr_learned_adam``)."""

    def __init__(self, params, lr=3e-3, betas=(0.9, 0.999), eps=1e-8, clip=2.0):
        self.params = params
        self.m = torch.zeros_like(params)
        self.v = torch.zeros_like(params)
        self.norm = torch.zeros(1, dtype=torch.float32, device=params.device)
        self.lr, self.betas, self.eps, self.clip = lr, betas, eps, clip
        self.t = 0

    def step(self, grad, lr=None):
        self.t += 1
        _lib.check(_lib.load().nsr_learned_adam(_ptr(self.params), _ptr(grad), _ptr(self.m), _ptr(self.v),
                                                self.params.numel(), self.t, float(lr or self.lr), self.betas[0],
                                                self.betas[1], self.eps, float(self.clip), _ptr(self.norm),
                                                _stream()))


def training_media(n_media, nz, nx, seed0=100, device=None):
    """Seeded breast-like training media (the record family of the benchmark, smaller grids)."""
    from .media import breast_record
    out = []
    for k in range(n_media):
        rec = breast_record(seed=seed0 + k, nz=nz, nx=nx, n_rx=min(192, nx // 4 - 8), rx_pitch=4)
        out.append((rec, Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=device)))
    return out


def train(steps=4000, nz=256, nx=384, batch=4, krylov_steps=48, lr=3e-3, n_media=16, channel_weight=1.0, seed=0,
          device=None, log=print, params=None, precision="fp32"):
    """Train the learned preconditioner on seeded breast-like media (GPU).

    Each step draws one training medium and ``batch`` (frequency, angle)
    systems from the benchmark's band (4.0-8.9 MHz, -25..25 degrees), whose
    receiver targets come from this solver's converged solves, and applies one
    clipped Adam step (cosine learning-rate decay to lr/10, as
    nsrno/train_dense_wave.py:38 schedules it)."""
    from .media import breast_bins
    device = torch.device(device or "cuda")
    rng = np.random.default_rng(seed)
    media = training_media(n_media, nz, nx, device=device)
    bins = breast_bins()
    net = LearnedPreconditioner(params, device=device, precision=precision)
    opt = Adam(net.params, lr=lr)
    history = []
    started = time.perf_counter()
    for step in range(steps):
        rec, med = media[step % len(media)]
        f = rng.choice(bins, size=batch, replace=False)
        th = np.deg2rad(rng.uniform(-25.0, 25.0, size=batch))
        bt = make_batch(med, f, th, with_target=channel_weight > 0)
        loss, grad, _ = loss_and_grad(net.params, bt, krylov_steps, channel_weight, precision=precision)
        if not math.isfinite(loss) or not bool(torch.isfinite(grad).all()):
            raise RuntimeError("non-finite training loss or gradient")
        cur = lr / 10 + 0.5 * (lr - lr / 10) * (1 + math.cos(math.pi * step / max(steps, 1)))
        opt.step(grad, lr=cur)
        history.append(loss)
        if step % 25 == 0 or step == steps - 1:
            log(json.dumps({"step": step, "loss": round(loss, 4), "lr": cur,
                            "grad_norm": float(opt.norm), "shift": net.shift,
                            "seconds": round(time.perf_counter() - started, 1)}))
    net.meta = dict(steps=steps, grid=[nz, nx], batch=batch, krylov_steps=krylov_steps, lr=lr, n_media=n_media,
                    channel_weight=channel_weight, seed=seed, final_loss=float(np.mean(history[-50:])),
                    seconds=time.perf_counter() - started, precision=precision)
    return net, history


def evaluate(path=WEIGHTS, precision=None, systems=220, seed=2, tolerance=1e-6, device=None):
    """BiCGSTAB iterations of the learned preconditioner on a held-out medium:
    the 1024 (x) x 768 (z) breast record of ``seed`` (seed 2 is the benchmark
    medium; training uses seeds 100 and up), ``systems`` (frequency, angle)
    systems spread evenly over its band, solved from zero to the FP64 true
    relative residual ``tolerance``.  Returns a dict with the mean and largest
    iteration counts and the number converged."""
    from .media import breast_record
    from .solver import solve_batched
    device = torch.device(device or "cuda")
    rec = breast_record(seed=seed)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=device)
    net = LearnedPreconditioner.load(path, device=device, precision=precision)
    f, a = rec.systems()
    pick = np.linspace(0, len(f) - 1, min(systems, len(f))).round().astype(int)
    f, a = f[pick], a[pick]
    setup = net.setup(med, np.unique(f))
    r = solve_batched(med, f, a, tolerance=tolerance, learned=setup)
    it = r.iterations.cpu().numpy()
    return {"weights": str(path), "precision": net.precision, "systems": int(len(f)),
            "converged": int(sum(x == "converged" for x in r.reasons())),
            "iterations_mean": float(it.mean()), "iterations_max": int(it.max())}


def main():
    ap = argparse.ArgumentParser(description="Train the learned preconditioner on the GPU")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--nz", type=int, default=256)
    ap.add_argument("--nx", type=int, default=384)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--krylov-steps", type=int, default=48)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--media", type=int, default=16)
    ap.add_argument("--channel-weight", type=float, default=1.0)
    ap.add_argument("--precision", choices=["fp32", "bf16"], default="fp32")
    ap.add_argument("--init", type=Path, default=None, help="start from these weights (fine-tuning)")
    ap.add_argument("--out", type=Path, default=WEIGHTS)
    ap.add_argument("--evaluate", type=Path, default=None,
                    help="no training: report the iterations these weights take on the held-out benchmark medium")
    ap.add_argument("--systems", type=int, default=220, help="systems of the evaluation")
    a = ap.parse_args()
    if a.evaluate is not None:
        print(json.dumps(evaluate(a.evaluate, precision=a.precision, systems=a.systems)))
        return
    init = None
    if a.init is not None:
        with np.load(a.init) as z:
            init = z["params"]
    net, _ = train(steps=a.steps, nz=a.nz, nx=a.nx, batch=a.batch, krylov_steps=a.krylov_steps, lr=a.lr,
                   n_media=a.media, channel_weight=a.channel_weight, params=init, precision=a.precision)
    net.save(a.out)
    print(json.dumps({"saved": str(a.out), **net.meta}))


if __name__ == "__main__":
    main()
