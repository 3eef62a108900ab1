"""Seeded synthetic records: grid, acquisition and (c, rho, alpha) media.

The reference ships no data for this path (its V5 records and checkpoints are
external).  These generators produce the two record families the solver is
measured and checked on:

* ``blob_record``   -- 256 x 256 nodes at 0.1 mm, 20-node PML, homogeneous
  water background with six Gaussian inclusions, alpha 0.5 dB/cm/MHz^1.1,
  plane waves at -15/0/+15 degrees and 1.0/1.5 MHz, 192 receivers.
* ``breast_record`` -- 768 (z) x 1024 (x) nodes at 0.05 mm, elliptical fat and
  glandular regions plus ten inclusions, alpha 0.4-1.0 dB/cm/MHz^1.1 per region,
  a 1 mm water coupling layer under the array, 11 angles in [-25, 25] degrees
  x 294 bins ``f = k 40 MHz / 2401`` (k = 241..534, 4.015-8.896 MHz), 192
  receivers at 0.2 mm pitch.

Material contrast vanishes inside the PML (the reference Solver validates the
same, theranostic/wave.py:170).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

WATER_C = 1500.0
WATER_RHO = 1000.0


@dataclass
class Record:
    """One acquisition record: a medium on a grid and its (frequency, angle) systems."""

    nz: int
    nx: int
    h: float
    n_pml: int
    face: int
    rx_cols: np.ndarray
    aperture_half_width: float
    c: np.ndarray
    rho: np.ndarray
    alpha: np.ndarray
    frequencies: np.ndarray
    angles: np.ndarray
    c0: float = WATER_C
    rho0: float = WATER_RHO
    pml_strength: float = 12.0
    alpha_power: float = 1.1
    name: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.nz * self.nx

    def systems(self):
        """All (frequency, angle) pairs, frequency-major (angles of one frequency adjacent)."""
        f = np.repeat(self.frequencies, len(self.angles))
        a = np.tile(self.angles, len(self.frequencies))
        return f, a

    def axes(self):
        x = (np.arange(self.nx) - (self.nx - 1) / 2.0) * self.h
        z = np.arange(self.nz) * self.h
        return x, z

    def interior(self):
        """Boolean [nz, nx]: nodes outside the PML."""
        m = np.zeros((self.nz, self.nx), dtype=bool)
        p = self.n_pml
        m[p:self.nz - p, p:self.nx - p] = True
        return m


def _centred_receivers(nx, count, pitch):
    centre = (nx - 1) / 2.0
    return np.round(centre + (np.arange(count) - (count - 1) / 2.0) * pitch).astype(np.int64)


def _taper(nz, nx, n_pml, ramp):
    """1 in the interior, 0 in the PML, a raised-cosine ramp of ``ramp`` nodes between."""
    def axis(n):
        i = np.arange(n)
        d = np.minimum(i - n_pml, n - 1 - n_pml - i).astype(np.float64)
        w = np.clip(d / ramp, 0.0, 1.0)
        return 0.5 - 0.5 * np.cos(math.pi * w)
    return axis(nz)[:, None] * axis(nx)[None, :]


def blob_record(seed=1, nz=256, nx=256, h=1e-4, n_pml=20, frequencies=(1.0e6, 1.5e6),
                angles_deg=(-15.0, 0.0, 15.0), n_blobs=6, alpha_db=0.5, n_rx=192, rx_pitch=1):
    rng = np.random.default_rng(seed)
    x, z = (np.arange(nx) - (nx - 1) / 2.0) * h, np.arange(nz) * h
    xx, zz = np.meshgrid(x, z)
    face = n_pml + 2
    dc = np.zeros((nz, nx))
    drho = np.zeros((nz, nx))
    lo_x, hi_x = x[n_pml], x[nx - 1 - n_pml]
    lo_z, hi_z = z[face + 8], z[nz - 1 - n_pml]
    for _ in range(n_blobs):
        cx, cz = rng.uniform(lo_x, hi_x), rng.uniform(lo_z, hi_z)
        cb, rb = rng.uniform(1400.0, 1600.0), rng.uniform(950.0, 1100.0)
        radius = rng.uniform(2e-3, 6e-3)
        g = np.exp(-((xx - cx) ** 2 + (zz - cz) ** 2) / radius ** 2)
        dc += (cb - WATER_C) * g
        drho += (rb - WATER_RHO) * g
    w = _taper(nz, nx, n_pml, 8)
    c = WATER_C + dc * w
    rho = WATER_RHO + drho * w
    alpha = np.full((nz, nx), alpha_db)
    rx = _centred_receivers(nx, n_rx, rx_pitch)
    return Record(nz=nz, nx=nx, h=h, n_pml=n_pml, face=face, rx_cols=rx,
                  aperture_half_width=n_rx * rx_pitch * h / 2.0,
                  c=c.astype(np.float32), rho=rho.astype(np.float32), alpha=alpha.astype(np.float32),
                  frequencies=np.asarray(frequencies, dtype=np.float64),
                  angles=np.deg2rad(np.asarray(angles_deg, dtype=np.float64)),
                  name=f"blobs{nz}x{nx}")


def breast_bins():
    """Frequency bins of the V5 clock: ``k * 40 MHz / 2401`` for k = 241..534."""
    k = np.arange(241, 535)
    return k * 40e6 / 2401.0


def breast_record(seed=2, nz=768, nx=1024, h=5e-5, n_pml=24, n_angles=11, bins=None,
                  n_inclusions=10, n_rx=192, rx_pitch=4):
    rng = np.random.default_rng(seed)
    x, z = (np.arange(nx) - (nx - 1) / 2.0) * h, np.arange(nz) * h
    xx, zz = np.meshgrid(x, z)
    face = n_pml + 4
    coupling = face + int(round(1e-3 / h))            # 1 mm water under the array
    c = np.full((nz, nx), WATER_C)
    rho = np.full((nz, nx), WATER_RHO)
    alpha = np.full((nz, nx), 0.002)
    z_top, z_bot = z[coupling], z[nz - 1 - n_pml - 8]
    x_half = x[nx - 1 - n_pml - 8]
    # Fat ellipse touching the coupling layer, glandular ellipse inside it.
    ez0, erz, erx = 0.5 * (z_top + z_bot), 0.5 * (z_bot - z_top), x_half * 0.95
    fat = ((xx / erx) ** 2 + ((zz - ez0) / erz) ** 2) <= 1.0
    c[fat], rho[fat], alpha[fat] = rng.uniform(1420, 1480), rng.uniform(920, 960), rng.uniform(0.4, 1.0)
    gz0, grz, grx = ez0 + 0.1 * erz, 0.55 * erz, 0.6 * erx
    gx0 = rng.uniform(-0.15, 0.15) * erx
    gland = (((xx - gx0) / grx) ** 2 + ((zz - gz0) / grz) ** 2) <= 1.0
    c[gland], rho[gland], alpha[gland] = rng.uniform(1500, 1560), rng.uniform(1020, 1060), rng.uniform(0.4, 1.0)
    for _ in range(n_inclusions):
        while True:
            cx, cz = rng.uniform(-erx, erx), rng.uniform(z_top, z_bot)
            if (cx / erx) ** 2 + ((cz - ez0) / erz) ** 2 < 0.8:
                break
        r = rng.uniform(0.5e-3, 3e-3)
        inc = ((xx - cx) ** 2 + (zz - cz) ** 2) <= r ** 2
        c[inc], rho[inc], alpha[inc] = rng.uniform(1420, 1560), rng.uniform(920, 1060), rng.uniform(0.4, 1.0)
    bins = breast_bins() if bins is None else np.asarray(bins, dtype=np.float64)
    angles = np.deg2rad(np.linspace(-25.0, 25.0, n_angles))
    rx = _centred_receivers(nx, n_rx, rx_pitch)
    return Record(nz=nz, nx=nx, h=h, n_pml=n_pml, face=face, rx_cols=rx,
                  aperture_half_width=n_rx * rx_pitch * h / 2.0,
                  c=c.astype(np.float32), rho=rho.astype(np.float32), alpha=alpha.astype(np.float32),
                  frequencies=bins, angles=angles, name=f"breast{nz}x{nx}")


def perturbed(record: Record, seed=3, dlogc=0.01, dlogrho=0.005, window=8e-3):
    """Copy of ``record`` with +dlogc / +dlogrho inside a seeded square window."""
    rng = np.random.default_rng(seed)
    x, z = record.axes()
    inner = record.interior()
    zi, xi = np.nonzero(inner)
    k = rng.integers(len(zi))
    cx, cz = x[xi[k]], z[zi[k]]
    xx, zz = np.meshgrid(x, z)
    win = (np.abs(xx - cx) <= window / 2) & (np.abs(zz - cz) <= window / 2) & inner
    out = Record(**{**record.__dict__})
    out.c = (record.c * np.where(win, math.exp(dlogc), 1.0)).astype(np.float32)
    out.rho = (record.rho * np.where(win, math.exp(dlogrho), 1.0)).astype(np.float32)
    return out
