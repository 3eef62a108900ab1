"""CPU oracle of the 8th-order dense operator -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module.  It restates in complex128 NumPy the
operator that the reference's dense path evaluates with FFTs on a padded grid:

* ``FrequencyGeometry``           nsrno/conditioned_wave.py:12-50  -> :class:`DenseGeometry`
* ``ConditionedFrequencySystem``  nsrno/conditioned_wave.py:52-80  -> :class:`DenseSystem`
* ``projected_operator``          nsrno/dense_wave.py:66-68        -> :meth:`DenseSystem.apply`
* ``adjoint_operator``            nsrno/dense_wave.py:70-82        -> :meth:`DenseSystem.adjoint`

It is pinned to golden vectors produced by the reference itself
(``tests/golden/reference_dense.npz``).
"""
from __future__ import annotations

import cmath
import math

import numpy as np

C0 = 1540.0
RHO0 = 1000.0
COEFF = (1225 / 1024, -245 / 3072, 49 / 5120, -5 / 7168)


class DenseGeometry:
    """Padded grid, staggered symbols, mask and PML profiles (conditioned_wave.py:12-50)."""

    def __init__(self, spec):
        self.spec = spec
        self.h, self.w = spec["medium_shape"][-2:]
        self.dx = spec["dx_m"]
        self.H = math.ceil((self.h + 64) / 32) * 32
        self.W = math.ceil((self.w + 64) / 32) * 32
        if "fft_shape" in spec:
            self.H, self.W = spec["fft_shape"]
        self.pz = (self.H - self.h) // 2
        self.px = (self.W - self.w) // 2
        qx = 2 * np.pi * np.fft.fftfreq(self.W)
        qz = 2 * np.pi * np.fft.fftfreq(self.H)
        self.Dx = self.symbol(qx)[None, :]
        self.Dz = self.symbol(qz)[:, None]
        self.mask = np.zeros((self.H, self.W))
        self.mask[self.pz:self.pz + self.h, self.px:self.px + self.w] = 1.0
        self.dt = spec["native_dt_s"]
        self.pml = spec["pml"]
        xx = np.arange(self.W) - self.px
        zz = np.arange(self.H) - self.pz
        self.arx = (1 - self.dt * self.damping(xx, self.w, 0.0))[None, :]
        self.arz = (1 - self.dt * self.damping(zz, self.h, 0.0))[:, None]
        self.avx = (1 - self.dt * self.damping(xx, self.w, 0.5))[None, :]
        self.avz = (1 - self.dt * self.damping(zz, self.h, 0.5))[:, None]

    def symbol(self, q):
        """Fourier symbol of the 8th-order staggered forward derivative."""
        return 2j * sum(a * np.sin((j + 0.5) * q) for j, a in enumerate(COEFF)) * np.exp(0.5j * q) / self.dx

    def damping(self, pos, size, stagger):
        pos = pos.astype(np.float64)
        left = np.where(pos < self.pml, (1 - (pos + stagger) / self.pml) ** 4, 0.0)
        right = np.where(pos >= size - self.pml, (1 - (size - 1 - pos - stagger) / self.pml) ** 4, 0.0)
        return (left + right) * 2 * C0 / self.dx

    def coefficients(self, m):
        """Crop the PML rim, replicate it back, replicate-pad to the FFT grid."""
        p = self.pml
        m = np.asarray(m, dtype=np.float64)
        m = np.pad(m[..., p:-p, p:-p], [(0, 0)] * (m.ndim - 2) + [(p, p), (p, p)], mode="edge")
        pad = [(0, 0)] * (m.ndim - 2) + [(self.pz, self.H - self.h - self.pz), (self.px, self.W - self.w - self.px)]
        return np.pad(m, pad, mode="edge")


class DenseSystem:
    """Coefficients of one medium at one frequency (conditioned_wave.py:53-69)."""

    def __init__(self, g: DenseGeometry, medium, alpha, frequency):
        self.g = g
        self.frequency = float(frequency)
        c, rho = g.coefficients(medium)
        self.c, self.rho = c, rho
        self.alpha = g.coefficients(np.asarray(alpha)[None])[0]
        self.a = RHO0 / rho
        self.D = cmath.exp(2j * math.pi * frequency * g.dt)
        self.q = 1 / self.D
        self.k0 = 2 * math.sin(math.pi * frequency * g.dt) / (g.dt * C0)
        ae = np.roll(self.a, -1, -1)
        az_ = np.roll(self.a, -1, -2)
        self.ax = 2 * self.a * ae / (self.a + ae) * g.mask
        self.az = 2 * self.a * az_ / (self.a + az_) * g.mask
        eta = [self.alpha * self.c / C0 * v for v in g.spec["eta_per_unit_alpha"]]
        amplitude = (1 + (eta[0] + eta[1]) / 2) ** 2
        hsum = sum(e / (amplitude * (1 + t * (self.D - 1) / g.dt)) for e, t in zip(eta, g.spec["taus_s"]))
        modulus = amplitude * (1 - hsum) / (1 - (1 - self.q) * hsum)
        self.mass = self.a * (C0 / self.c) ** 2 / modulus
        self.svx = (self.D - 1) / (self.D - g.avx)
        self.svz = (self.D - 1) / (self.D - g.avz)
        self.gvx = 1 + (1 - g.avx) * self.q
        self.gvz = 1 + (1 - g.avz) * self.q
        self.mx = (g.arx != 1).astype(np.float64)
        self.mz = (g.arz != 1).astype(np.float64)

    def _call(self, p):
        g = self.g
        ifft2, fft2 = np.fft.ifft2, np.fft.fft2
        spectrum = fft2(p)
        x = self.ax * self.svx * ifft2(g.Dx * spectrum)
        z = self.az * self.svz * ifft2(g.Dz * spectrum)

        def part(flux, gain, mask, ar, symbol):
            regular = ifft2(-np.conj(symbol) * fft2(flux))
            provisional = ifft2(-np.conj(symbol) * fft2(gain * flux))
            return mask / (self.D - ar) * regular + (1 + (1 - mask) / (self.D - ar)) * provisional

        spatial = (self.D - 1) / self.D / self.k0 ** 2 * (part(x, self.gvx, self.mx, g.arx, g.Dx) +
                                                         part(z, self.gvz, self.mz, g.arz, g.Dz))
        return g.mask * (spatial + self.mass * p) + (1 - g.mask) * p

    def apply(self, p):
        """Projected operator ``mask A(mask p) + (1 - mask) p`` (dense_wave.py:66-68)."""
        m = self.g.mask
        return m * self._call(m * p) + (1 - m) * p

    def adjoint(self, p):
        """Analytic adjoint of :meth:`apply` (dense_wave.py:70-82)."""
        g = self.g
        ifft2, fft2 = np.fft.ifft2, np.fft.fft2
        y = g.mask * p
        scalar = (self.D - 1) / self.D / self.k0 ** 2
        weighted = np.conj(scalar) * y

        def axis(ax, sv, gain, mask, ar, symbol):
            left = mask / (self.D - ar)
            right = 1 + (1 - mask) / (self.D - ar)
            first = ifft2(-symbol * fft2(np.conj(left) * weighted))
            second = ifft2(-symbol * fft2(np.conj(right) * weighted))
            flux = np.conj(ax * sv) * (first + np.conj(gain) * second)
            return ifft2(np.conj(symbol) * fft2(flux))

        value = (axis(self.ax, self.svx, self.gvx, self.mx, g.arx, g.Dx) +
                 axis(self.az, self.svz, self.gvz, self.mz, g.arz, g.Dz) + np.conj(self.mass) * y)
        return g.mask * value + (1 - g.mask) * p

    def fixed_preconditioner(self, p, shift=0.15, adjoint=False):
        """``mask IFFT(FFT(p) / (1 + lap/k0^2 - i shift))`` (conditioned_wave.py:90-92);
        the adjoint solve conjugates the multiplier (dense_wave.py:195)."""
        g = self.g
        lap = -(np.abs(g.Dx) ** 2 + np.abs(g.Dz) ** 2)
        m = 1.0 / (1.0 + lap / self.k0 ** 2 - 1j * shift)
        if adjoint:
            m = np.conj(m)
        return g.mask * np.fft.ifft2(m * np.fft.fft2(p))

    def source(self, line):
        """Pressure source of a line on the array row (conditioned_wave.py:82-88)."""
        g = self.g
        zi, xi = g.spec["source_c_lookup_zx"]
        source_c = self.c[zi + g.pz, xi + g.px]
        line = np.atleast_2d(line)
        profile = np.zeros((line.shape[0], g.H, g.W), dtype=np.complex128)
        face = round(-g.spec["z0_m"] / g.dx) + g.pz
        profile[:, face, g.px:g.px + line.shape[-1]] = line
        return profile * self.a * C0 ** 2 * 2 * g.dt / (source_c * g.dx * (self.D - 1))


def homogeneous(g: DenseGeometry, frequency):
    """The uniform reference medium of the dense acquisition (dense_wave.py:53-55)."""
    medium = np.stack((np.full((g.h, g.w), C0), np.full((g.h, g.w), RHO0)))
    return DenseSystem(g, medium, np.full((g.h, g.w), 0.002), frequency)


def assemble(system: DenseSystem, reference: DenseSystem, line, pref):
    """``S(src) - S0(src) - A p_ref + A0 p_ref`` (dense_wave.py:46-57), pref [n, H, W]."""
    out = system.source(line) - reference.source(line)
    for k in range(pref.shape[0]):
        out[k] += -system.apply(pref[k]) + reference.apply(pref[k])
    return out
