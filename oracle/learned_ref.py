"""CPU oracle of the learned preconditioner -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU leg of ``bench.py`` may
import this module, and only to check results.  The product path
(``nsrno_b200``) never imports it.

It restates, in float64 / complex128 PyTorch on the CPU (autograd supplies the
reference gradients the hand-written backward kernels are checked against),
the reference's ``LearnedPreconditioner`` (nsrno/conditioned_wave.py:94-117)
and ``learned_apply`` (nsrno/dense_wave.py:150-165) on the 5-point grid:

* context ``(log(c/1540)/.06, log(rho/1000)/.08, log1p(alpha), f/6e6 - 1, mask)``
  (conditioned_wave.py:105-106), 8x average pooled (:107);
* three 3x3 convolutions 5->16->16->4 with tanh between (:97-98);
* bilinear upsampling to the grid, ``align_corners=False`` (:108);
* diagonal gains ``(1 + tanh(m0)/2) exp(i tanh(m1)/2)`` (inner) and the same of
  m2, m3 (outer) (:109-110);
* the spectral multiplier ``exp(tanh(mod0)/2 + i tanh(mod1)/2) / (1 - q2 - i s)``
  with ``q2 = -lap/k0^2``, ``angular = |Dx|^2/(-lap + 1)``, the basis
  ``(1, q2/(1+q2), angular, angular q2/(1+q2))`` and ``s = clamp(exp(log_shift),
  .01, 1)`` (:112-115);
* ``apply(r) = outer * ifft2(multiplier * fft2(inner * r))`` (:116) and its
  exact adjoint (dense_wave.py:163-164).

Mapping onto the 5-point path (stated once, used everywhere):

* ``lap`` and ``Dx`` are the symbols of the 5-point operator,
  ``-4 sin^2(q/2)/h^2`` per axis, instead of the 8th-order staggered ones of the
  dense grid; the mask is one everywhere (the 5-point grid has no FFT padding);
* the 5-point path uses the ``exp(-i omega t)`` convention (its operator is the
  complex conjugate of the dense one), so the preconditioner is the conjugate
  map ``M(r) = conj(M_ref(conj(r))) / (k0 h)^2``.  The ``1/(k0 h)^2`` factor
  puts it in the units of the h^2-scaled operator; with the network output
  zero, no spectral modulation and ``s = 0.15`` it is exactly the fixed
  shifted-Laplace preconditioner of the solver.

Parameters travel as one flat float32 vector in the order of the reference
module's ``state_dict``: ``spectral [2,4]``, ``log_shift``, ``context.0.weight
[16,5,3,3]``, ``context.0.bias``, ``context.2.weight [16,16,3,3]``,
``context.2.bias``, ``context.4.weight [4,16,3,3]``, ``context.4.bias`` -- 3645
numbers, the parameter count the reference documents for this network.
"""
from __future__ import annotations

import math

import numpy as np
import torch
from torch.nn import functional as F

C_REF = 1540.0       # nsrno/wave_operator.py:12 (C0), the context normalisation
RHO_REF = 1000.0     # nsrno/wave_operator.py:12 (RHO0)

SHAPES = [
    ("spectral", (2, 4)),
    ("log_shift", ()),
    ("context.0.weight", (16, 5, 3, 3)),
    ("context.0.bias", (16,)),
    ("context.2.weight", (16, 16, 3, 3)),
    ("context.2.bias", (16,)),
    ("context.4.weight", (4, 16, 3, 3)),
    ("context.4.bias", (4,)),
]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)   # 3645
N_SPECTRAL = 9                                       # spectral [2,4] and log_shift lead
N_CONV = N_PARAMS - N_SPECTRAL                       # 3636 network weights


def unflatten(flat):
    """Flat parameter vector -> dict of tensors (views of ``flat``)."""
    out, k = {}, 0
    for name, shape in SHAPES:
        m = int(np.prod(shape)) if shape else 1
        out[name] = flat[k:k + m].reshape(shape)
        k += m
    return out


def initial_parameters(seed=0):
    """Untrained parameters: torch's default conv initialisation for the first two
    layers, zeros for the last layer and the spectral weights, log(0.15)
    (conditioned_wave.py:99-101) -- the identity gains of the reference."""
    g = torch.Generator().manual_seed(seed)
    parts = []
    for name, shape in SHAPES:
        if name in ("context.0.weight", "context.2.weight"):
            fan_in = shape[1] * 9
            bound = 1.0 / math.sqrt(fan_in)
            parts.append((torch.rand(shape, generator=g, dtype=torch.float64) * 2 - 1).reshape(-1) * bound)
        elif name in ("context.0.bias", "context.2.bias"):
            fan_in = (5 if name == "context.0.bias" else 16) * 9
            bound = 1.0 / math.sqrt(fan_in)
            parts.append((torch.rand(shape, generator=g, dtype=torch.float64) * 2 - 1).reshape(-1) * bound)
        elif name == "log_shift":
            parts.append(torch.tensor([math.log(0.15)], dtype=torch.float64))
        else:
            parts.append(torch.zeros(int(np.prod(shape)), dtype=torch.float64))
    return torch.cat(parts)


def context(c, rho, alpha, frequency_hz):
    """Five context channels [5, nz, nx] (conditioned_wave.py:105-106, mask = 1)."""
    c = torch.as_tensor(c, dtype=torch.float64)
    rho = torch.as_tensor(rho, dtype=torch.float64)
    alpha = torch.as_tensor(alpha, dtype=torch.float64)
    return torch.stack(((c / C_REF).log() / 0.06, (rho / RHO_REF).log() / 0.08, torch.log1p(alpha),
                        torch.ones_like(c) * (frequency_hz / 6e6 - 1), torch.ones_like(c)))


def pool8(ctx):
    """8x8 average pool, floor mode (``F.avg_pool2d(context, 8)``)."""
    C, H, W = ctx.shape
    h, w = H // 8, W // 8
    return ctx[:, : 8 * h, : 8 * w].reshape(C, h, 8, w, 8).mean(dim=(2, 4))


def conv3x3(x, weight, bias):
    """3x3 cross-correlation with zero padding 1: x [Cin, h, w] -> [Cout, h, w]."""
    Cin, h, w = x.shape
    xp = F.pad(x, (1, 1, 1, 1))
    out = bias[:, None, None].expand(-1, h, w).clone()
    for ky in range(3):
        for kx in range(3):
            out = out + torch.einsum("oc,chw->ohw", weight[:, :, ky, kx], xp[:, ky:ky + h, kx:kx + w])
    return out


def network(params, pooled):
    """Low-resolution activations: (tanh layer 1, tanh layer 2, maps [4, h, w])."""
    p = unflatten(params)
    a1 = torch.tanh(conv3x3(pooled, p["context.0.weight"], p["context.0.bias"]))
    a2 = torch.tanh(conv3x3(a1, p["context.2.weight"], p["context.2.bias"]))
    maps = conv3x3(a2, p["context.4.weight"], p["context.4.bias"])
    return a1, a2, maps


def upsample_indices(n_in, n_out):
    """Bilinear source indices and weights of ``F.interpolate(..., align_corners=False)``
    for one axis: ``src = max((dst + .5) n_in/n_out - .5, 0)``."""
    scale = n_in / n_out
    src = np.maximum((np.arange(n_out) + 0.5) * scale - 0.5, 0.0)
    i0 = np.floor(src).astype(np.int64)
    i0 = np.minimum(i0, n_in - 1)
    i1 = np.minimum(i0 + 1, n_in - 1)
    l1 = src - i0
    return i0, i1, 1.0 - l1, l1


def upsample(maps, nz, nx):
    """Bilinear upsampling [C, h, w] -> [C, nz, nx] (conditioned_wave.py:108)."""
    _, h, w = maps.shape
    z0, z1, wz0, wz1 = upsample_indices(h, nz)
    x0, x1, wx0, wx1 = upsample_indices(w, nx)
    wz0, wz1 = torch.as_tensor(wz0)[:, None], torch.as_tensor(wz1)[:, None]
    wx0, wx1 = torch.as_tensor(wx0)[None, :], torch.as_tensor(wx1)[None, :]
    rows0 = maps[:, z0, :]
    rows1 = maps[:, z1, :]
    top = rows0[:, :, x0] * wx0 + rows0[:, :, x1] * wx1
    bot = rows1[:, :, x0] * wx0 + rows1[:, :, x1] * wx1
    return top * wz0 + bot * wz1


def gains(maps_full):
    """(inner, outer) complex [nz, nx] of the 5-point path: the conjugates of
    conditioned_wave.py:109-110."""
    t = torch.tanh(maps_full)
    inner = (1 + 0.5 * t[0]) * torch.exp(-0.5j * t[1])
    outer = (1 + 0.5 * t[2]) * torch.exp(-0.5j * t[3])
    return inner, outer


def symbols(nz, nx, h, frequency_hz, c0):
    """``(q2, angular, kh2)`` on the natural FFT grid [nz, nx] for the 5-point symbols."""
    k0 = 2 * math.pi * frequency_hz / c0
    qx = 2 * math.pi * torch.fft.fftfreq(nx, dtype=torch.float64)
    qz = 2 * math.pi * torch.fft.fftfreq(nz, dtype=torch.float64)
    dx2 = (4 * torch.sin(qx / 2) ** 2 / h ** 2)[None, :]
    dz2 = (4 * torch.sin(qz / 2) ** 2 / h ** 2)[:, None]
    lap = -(dx2 + dz2)
    q2 = -lap / k0 ** 2
    angular = (dx2 / (-lap + 1)).expand(nz, nx)
    return q2, angular, (k0 * h) ** 2


def multiplier(params, nz, nx, h, frequency_hz, c0):
    """Spectral multiplier of the 5-point path [nz, nx] (h^2 units, conjugate map)."""
    p = unflatten(params)
    q2, angular, kh2 = symbols(nz, nx, h, frequency_hz, c0)
    basis = torch.stack((torch.ones_like(q2), q2 / (1 + q2), angular, angular * q2 / (1 + q2)))
    mod = torch.einsum("ck,khw->chw", p["spectral"], basis)
    shift = p["log_shift"].exp().clamp(0.01, 1.0)
    ref = torch.exp(0.5 * torch.tanh(mod[0]) + 0.5j * torch.tanh(mod[1])) / (1 - q2 - 1j * shift)
    return ref.conj() / kh2


class Learned:
    """The learned preconditioner of one medium at one frequency."""

    def __init__(self, params, c, rho, alpha, frequency_hz, h, c0):
        c = torch.as_tensor(c, dtype=torch.float64)
        nz, nx = c.shape
        self.pooled = pool8(context(c, rho, alpha, frequency_hz))
        self.a1, self.a2, self.maps = network(params, self.pooled)
        self.maps_full = upsample(self.maps, nz, nx)
        self.inner, self.outer = gains(self.maps_full)
        self.mult = multiplier(params, nz, nx, h, frequency_hz, c0)

    def core(self, r, adjoint=False):
        m = self.mult.conj() if adjoint else self.mult
        return torch.fft.ifft2(m * torch.fft.fft2(r))

    def apply(self, r):
        return self.outer * self.core(self.inner * r)

    def adjoint(self, r):
        return self.inner.conj() * self.core(self.outer.conj() * r, adjoint=True)


def reference_map(ref_apply, r, kh2):
    """The conjugate map of the 5-point path applied to a reference apply function."""
    return ref_apply(r.conj()).conj() / kh2


class Stencil:
    """The h^2-scaled 5-point operator as five coefficient planes (torch, complex128)."""

    def __init__(self, csr, nz, nx, h):
        d = csr.diagonal(0) * h ** 2
        e = np.zeros(nz * nx, complex)
        e[:-1] = csr.diagonal(1) * h ** 2
        s = np.zeros(nz * nx, complex)
        s[:-nx] = csr.diagonal(nx) * h ** 2
        self.D = torch.tensor(d.reshape(nz, nx))
        self.E = torch.tensor(e.reshape(nz, nx))
        self.S = torch.tensor(s.reshape(nz, nx))

    def __call__(self, u, adjoint=False):
        D, E, S = (t.conj() for t in (self.D, self.E, self.S)) if adjoint else (self.D, self.E, self.S)
        y = D * u
        y = y + E * F.pad(u[:, 1:], (0, 1)) + F.pad((E * u)[:, :-1], (1, 0))
        y = y + S * F.pad(u[1:, :], (0, 0, 0, 1)) + F.pad((S * u)[:-1, :], (0, 0, 1, 0))
        return y


def mr_loss(operator, precondition, b, steps, rx=None, target=None):
    """Training objective: ``steps`` minimal-residual iterations from zero,

        z = M r,  w = A z,  g = <w, r>/<w, w>,  x += g z,  r -= g w,

    then ``log(|r|^2/|b|^2)`` plus, when ``target`` is given,
    ``log(|x[rx] - target|^2/|target|^2)`` (the relative receiver error of the
    warm field against the converged solve, the channel term of the
    reference's training loss, nsrno/train_dense_wave.py:19-21,66-68)."""
    r = b.clone()
    x = torch.zeros_like(b)
    for _ in range(steps):
        z = precondition(r)
        w = operator(z)
        g = (w.conj() * r).sum() / (w.conj() * w).sum()
        x = x + g * z
        r = r - g * w
    loss = torch.log(r.abs().square().sum() / b.abs().square().sum())
    if target is not None:
        d = x.reshape(-1)[rx]
        loss = loss + torch.log((d - target).abs().square().sum() / target.abs().square().sum())
    return loss
