"""The dense path's operator: 8th-order staggered derivatives, split PML and
two-relaxation attenuation on a padded grid (nsrno/conditioned_wave.py:12-80).

:class:`DenseGeometry` mirrors ``FrequencyGeometry`` (padded grid, native mask,
receiver columns, PML profiles); :class:`DenseSystem` mirrors
``ConditionedFrequencySystem`` (coefficients of one medium at one frequency)
and applies the projected operator or its adjoint with the direct-stencil
kernels of ``nsr_dense_apply``.  Coefficients are formed once per system on
the host in double precision and kept on the device.
"""
from __future__ import annotations

import cmath
import ctypes
import math

import numpy as np
import torch

from . import _lib

C0 = 1540.0      # reference speed of the dense path (nsrno/wave_operator.py:12)
RHO0 = 1000.0


def _damping(pos, size, n_pml, stagger, dx):
    """Quartic PML damping of the reference discretisation (conditioned_wave.py:32-36)."""
    pos = np.asarray(pos, dtype=np.float64)
    lo = np.where(pos < n_pml, (1.0 - (pos + stagger) / n_pml) ** 4, 0.0)
    hi = np.where(pos >= size - n_pml, (1.0 - (size - 1 - pos - stagger) / n_pml) ** 4, 0.0)
    return (lo + hi) * 2.0 * C0 / dx


class DenseGeometry:
    """Padded grid of a native ``[h, w]`` medium (conditioned_wave.py:13-31)."""

    def __init__(self, spec):
        self.spec = dict(spec)
        self.h, self.w = self.spec["medium_shape"][-2:]
        self.dx = float(self.spec["dx_m"])
        if "fft_shape" in self.spec:
            self.H, self.W = self.spec["fft_shape"]
            if self.H - self.h < 16 or self.W - self.w < 16:
                raise ValueError("padding must separate the 8th-order stencil support")
        else:
            self.H = math.ceil((self.h + 64) / 32) * 32
            self.W = math.ceil((self.w + 64) / 32) * 32
        self.pz = (self.H - self.h) // 2
        self.px = (self.W - self.w) // 2
        self.dt = float(self.spec["native_dt_s"])
        self.pml = int(self.spec["pml"])
        self.face = round(-self.spec["z0_m"] / self.dx) + self.pz
        self.rx_cols = np.round((np.arange(192) * 0.0002 - 0.0191 - self.spec["x0_m"]) / self.dx).astype(np.int64) + self.px
        cols = np.arange(self.W) - self.px
        rows = np.arange(self.H) - self.pz
        self.arx = 1.0 - self.dt * _damping(cols, self.w, self.pml, 0.0, self.dx)
        self.arz = 1.0 - self.dt * _damping(rows, self.h, self.pml, 0.0, self.dx)
        self.avx = 1.0 - self.dt * _damping(cols, self.w, self.pml, 0.5, self.dx)
        self.avz = 1.0 - self.dt * _damping(rows, self.h, self.pml, 0.5, self.dx)
        self.struct = _lib.NsrDenseGrid(self.H, self.W, self.pz, self.px, self.h, self.w, self.dx)

    def pad_material(self, m):
        """Crop the PML rim, replicate it back and replicate-pad to the padded grid (conditioned_wave.py:37-41)."""
        m = np.asarray(m, dtype=np.float64)
        p = self.pml
        inner = m[..., p:-p, p:-p]
        lead = [(0, 0)] * (m.ndim - 2)
        m = np.pad(inner, lead + [(p, p), (p, p)], mode="edge")
        return np.pad(m, lead + [(self.pz, self.H - self.h - self.pz), (self.px, self.W - self.w - self.px)],
                      mode="edge")

    def pad_field(self, p):
        return torch.nn.functional.pad(p, (self.px, self.W - self.w - self.px, self.pz, self.H - self.h - self.pz))


class DenseSystem:
    """One medium ``[2, h, w] = (c, rho)`` with attenuation ``alpha [h, w]`` at one frequency."""

    def __init__(self, geometry: DenseGeometry, medium, alpha, frequency, device="cuda"):
        g = geometry
        self.g = g
        self.frequency = float(frequency)
        medium = np.asarray(torch.as_tensor(medium).detach().cpu(), dtype=np.float64)
        alpha = np.asarray(torch.as_tensor(alpha).detach().cpu(), dtype=np.float64)
        if medium.shape != (2, g.h, g.w) or alpha.shape != (g.h, g.w):
            raise ValueError("Expected native [2,z,x] medium and [z,x] alpha")
        c, rho = g.pad_material(medium)
        al = g.pad_material(alpha)
        mask = np.zeros((g.H, g.W))
        mask[g.pz:g.pz + g.h, g.px:g.px + g.w] = 1.0
        a = RHO0 / rho
        D = cmath.exp(2j * math.pi * self.frequency * g.dt)
        q = 1.0 / D
        k0 = 2.0 * math.sin(math.pi * self.frequency * g.dt) / (g.dt * C0)
        # harmonic means on the faces n+1/2 (periodic neighbour, zero outside the mask)
        a_east = np.roll(a, -1, axis=1)
        a_south = np.roll(a, -1, axis=0)
        ax = 2.0 * a * a_east / (a + a_east) * mask
        az = 2.0 * a * a_south / (a + a_south) * mask
        # two-relaxation modulus (conditioned_wave.py:62-66)
        eta0, eta1 = (al * c / C0 * v for v in g.spec["eta_per_unit_alpha"])
        amp = (1.0 + 0.5 * (eta0 + eta1)) ** 2
        taus = g.spec["taus_s"]
        relax = eta0 / (amp * (1.0 + taus[0] * (D - 1.0) / g.dt)) + eta1 / (amp * (1.0 + taus[1] * (D - 1.0) / g.dt))
        modulus = amp * (1.0 - relax) / (1.0 - (1.0 - q) * relax)
        mass = a * (C0 / c) ** 2 / modulus

        def profiles(av, ar):
            sv = (D - 1.0) / (D - av)
            gv = 1.0 + (1.0 - av) * q
            m = (ar != 1.0).astype(np.float64)
            left = m / (D - ar)
            right = 1.0 + (1.0 - m) / (D - ar)
            return [sv, gv, left, right]

        px = profiles(g.avx, g.arx)
        pz = profiles(g.avz, g.arz)
        packed = np.concatenate([ax.ravel(), az.ravel(), mass.astype(np.complex128).view(np.float64).ravel()] +
                                [np.asarray(v, np.complex128).view(np.float64) for v in px] +
                                [np.asarray(v, np.complex128).view(np.float64) for v in pz])
        self.coef = torch.as_tensor(packed, dtype=torch.float64, device=device)
        nbytes = _lib.load().nsr_dense_coef_bytes(ctypes.byref(g.struct))
        if nbytes != self.coef.numel() * 8:
            raise RuntimeError("dense coefficient layout mismatch")
        self.D, self.q, self.k0 = D, q, k0
        self.scal = (D - 1.0) / D / k0 ** 2
        self.c, self.rho, self.alpha = c, rho, al

    def _run(self, p, adjoint):
        g = self.g
        p = torch.as_tensor(p)
        squeeze = p.dim() == 2
        if squeeze:
            p = p[None]
        if p.dim() != 3 or tuple(p.shape[1:]) != (g.H, g.W):
            raise ValueError(f"fields must be [n, {g.H}, {g.W}]")
        if not p.is_cuda:
            raise ValueError("fields must be CUDA tensors (no CPU path)")
        if p.dtype not in (torch.complex64, torch.complex128):
            p = p.to(torch.complex128)
        p = p.contiguous()
        prec = 1 if p.dtype == torch.complex128 else 0
        lib = _lib.load()
        nbytes = lib.nsr_dense_workspace_size(ctypes.byref(g.struct), p.shape[0], prec)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=p.device)
        y = torch.empty_like(p)
        _lib.check(lib.nsr_dense_apply(ctypes.byref(g.struct), ctypes.c_void_p(self.coef.data_ptr()),
                                       float(self.scal.real), float(self.scal.imag), p.shape[0], int(adjoint), prec,
                                       ctypes.c_void_p(p.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                       ctypes.c_void_p(ws.data_ptr()), nbytes,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return y[0] if squeeze else y

    def apply(self, p):
        """``mask A(mask p) + (1 - mask) p`` (nsrno/dense_wave.py:66-68)."""
        return self._run(p, False)

    def adjoint(self, p):
        """Its exact adjoint (nsrno/dense_wave.py:70-82)."""
        return self._run(p, True)
