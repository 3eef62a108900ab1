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
        # 192 receivers at 0.2 mm from x = -19.1 mm (nsrno/conditioned_wave.py:30); a spec may
        # describe another array with rx_count, rx_pitch_m and rx_first_m
        count = int(self.spec.get("rx_count", 192))
        pitch = float(self.spec.get("rx_pitch_m", 0.0002))
        first = float(self.spec.get("rx_first_m", -0.0191))
        self.rx_cols = np.round((np.arange(count) * pitch + first - self.spec["x0_m"]) / self.dx).astype(np.int64) + self.px
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

    def pad_material_t(self, m):
        """:meth:`pad_material` in torch (differentiable): ``m [k, h, w]`` -> ``[k, H, W]``."""
        F = torch.nn.functional
        p = self.pml
        inner = m[:, p:-p, p:-p]
        m = F.pad(inner[None], (p, p, p, p), mode="replicate")
        return F.pad(m, (self.px, self.W - self.w - self.px, self.pz, self.H - self.h - self.pz),
                     mode="replicate")[0]

    def mask_t(self, device):
        mask = torch.zeros((self.H, self.W), dtype=torch.float64, device=device)
        mask[self.pz:self.pz + self.h, self.px:self.px + self.w] = 1.0
        return mask


def medium_terms(g: DenseGeometry, medium, alpha, frequency):
    """The medium-dependent terms of the dense operator at one frequency, in
    torch float64 (differentiable w.r.t. ``medium [2, h, w] = (c, rho)``):
    padded c and rho, a = rho0/rho, the face coefficients ax, az (harmonic
    means with the periodic neighbour, zero outside the mask) and the
    two-relaxation mass term (nsrno/conditioned_wave.py:53-69)."""
    c, rho = g.pad_material_t(medium).unbind(0)
    al = g.pad_material_t(alpha[None])[0]
    mask = g.mask_t(medium.device)
    f = float(frequency)
    D = cmath.exp(2j * math.pi * f * g.dt)
    q = 1.0 / D
    a = RHO0 / rho
    a_east = torch.roll(a, -1, dims=1)
    a_south = torch.roll(a, -1, dims=0)
    ax = 2.0 * a * a_east / (a + a_east) * mask
    az = 2.0 * a * a_south / (a + a_south) * mask
    eta0, eta1 = (al * c / C0 * v for v in g.spec["eta_per_unit_alpha"])
    amp = (1.0 + 0.5 * (eta0 + eta1)) ** 2
    taus = g.spec["taus_s"]
    relax = eta0 / (amp * (1.0 + taus[0] * (D - 1.0) / g.dt)) + eta1 / (amp * (1.0 + taus[1] * (D - 1.0) / g.dt))
    modulus = amp * (1.0 - relax) / (1.0 - (1.0 - q) * relax)
    mass = a * (C0 / c) ** 2 / modulus
    return dict(c=c, rho=rho, alpha=al, a=a, ax=ax, az=az, mass=mass, mask=mask, D=D, q=q)


def source_term(g: DenseGeometry, terms, line):
    """Pressure source of lines ``[n, w]`` on the array row (nsrno/conditioned_wave.py:82-88),
    differentiable through ``terms`` (a and the source speed)."""
    zi, xi = g.spec["source_c_lookup_zx"]
    source_c = terms["c"][zi + g.pz, xi + g.px]
    dtype = torch.complex128 if line.dtype in (torch.complex128, torch.float64) else torch.complex64
    profile = torch.zeros((line.shape[0], g.H, g.W), dtype=dtype, device=line.device)
    profile[:, g.face, g.px:g.px + line.shape[-1]] = line.to(dtype)
    scale = C0 ** 2 * 2 * g.dt / (g.dx * (terms["D"] - 1.0))
    return profile * (terms["a"] * scale / source_c).to(dtype)


class DenseSystem:
    """One medium ``[2, h, w] = (c, rho)`` with attenuation ``alpha [h, w]`` at one frequency."""

    def __init__(self, geometry: DenseGeometry, medium, alpha, frequency, device="cuda"):
        g = geometry
        self.g = g
        self.frequency = float(frequency)
        medium = torch.as_tensor(medium).detach().to(device=device, dtype=torch.float64)
        alpha = torch.as_tensor(alpha).detach().to(device=device, dtype=torch.float64)
        if tuple(medium.shape) != (2, g.h, g.w) or tuple(alpha.shape) != (g.h, g.w):
            raise ValueError("Expected native [2,z,x] medium and [z,x] alpha")
        with torch.no_grad():
            terms = medium_terms(g, medium, alpha, self.frequency)
        self.terms = terms
        D, q = terms["D"], terms["q"]
        k0 = 2.0 * math.sin(math.pi * self.frequency * g.dt) / (g.dt * C0)
        ax = terms["ax"].cpu().numpy()
        az = terms["az"].cpu().numpy()
        mass = terms["mass"].cpu().numpy()

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
        self.c, self.rho, self.alpha = (terms[k].cpu().numpy() for k in ("c", "rho", "alpha"))

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

    # ------------------------------------------------------------------
    # Preconditioner, source and assembly (nsrno/conditioned_wave.py:82-92,
    # nsrno/dense_wave.py:46-62)
    # ------------------------------------------------------------------
    def fixed_preconditioner(self, shift=0.15, adjoint=False):
        """``r -> mask IFFT(FFT(r) / (1 + lap/k0^2 - i shift))`` (conditioned_wave.py:90-92) on the
        device (``nsr_dense_precondition``); ``adjoint`` conjugates the multiplier as
        nsrno/dense_wave.py:195 does for the adjoint solve.  Complex64 arithmetic."""
        g = self.g
        k0dx2 = (self.k0 * g.dx) ** 2

        def apply(r):
            r = torch.as_tensor(r)
            squeeze = r.dim() == 2
            x = (r[None] if squeeze else r).to(torch.complex64).contiguous()
            if not x.is_cuda or tuple(x.shape[1:]) != (g.H, g.W):
                raise ValueError(f"fields must be CUDA [n, {g.H}, {g.W}]")
            lib = _lib.load()
            nbytes = lib.nsr_dense_precondition_workspace_size(ctypes.byref(g.struct), x.shape[0])
            if nbytes == 0:
                raise ValueError("the dense preconditioner needs H and W in [8, 2048] with no prime factor above 61")
            ws = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
            y = torch.empty_like(x)
            _lib.check(lib.nsr_dense_precondition(ctypes.byref(g.struct), float(k0dx2), float(shift), x.shape[0],
                                                  int(bool(adjoint)), ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                                                  nbytes, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
            y = y.to(r.dtype)
            return y[0] if squeeze else y
        return apply

    def source(self, line):
        """Pressure source of a line on the array row (conditioned_wave.py:82-88):
        ``line [n, w]`` padded into row ``face``, times ``a c0^2 2 dt / (c_src dx (D - 1))``."""
        line = torch.as_tensor(line)
        squeeze = line.dim() == 1
        if squeeze:
            line = line[None]
        terms = {k: (v.to(line.device) if torch.is_tensor(v) else v) for k, v in self.terms.items()}
        out = source_term(self.g, terms, line)
        return out[0] if squeeze else out


def homogeneous_system(geometry: DenseGeometry, frequency, device="cuda"):
    """The uniform reference medium (1540 m/s, 1000 kg/m^3, alpha 0.002) of the
    dense acquisition (nsrno/dense_wave.py:53-55)."""
    medium = np.stack((np.full((geometry.h, geometry.w), C0), np.full((geometry.h, geometry.w), RHO0)))
    return DenseSystem(geometry, medium, np.full((geometry.h, geometry.w), 0.002), frequency, device=device)


def assemble(system: DenseSystem, reference: DenseSystem, line, pref):
    """Scattered-field right-hand side with homogeneous-reference subtraction
    (nsrno/dense_wave.py:46-57): ``S(src) - S0(src) - A p_ref + A0 p_ref``."""
    return system.source(line) - reference.source(line) - system.apply(pref) + reference.apply(pref)


def solve(system: DenseSystem, rhs, adjoint=False, tolerance=1e-5, restart=24, max_cycles=100, shift=0.15,
          initial=None):
    """Converged dense-path solve of ``A x = rhs`` (or ``A^H x = rhs``): the
    GMRES branch of ``solve_system`` (nsrno/dense_wave.py:212-225) with the
    fixed preconditioner, run on the device by ``nsr_dense_solve`` -- all
    fields (angles) as one vector, complex64 Krylov vectors with FP64 inner
    products and Givens recurrence, a complex128 iterate and an FP64 true
    residual at every restart.  ``rhs`` is ``[n, H, W]`` or ``[H, W]``.
    Returns ``(x, info)`` with the reference's info keys."""
    import time
    started = time.perf_counter()
    g = system.g
    rhs = torch.as_tensor(rhs)
    squeeze = rhs.dim() == 2
    b = (rhs[None] if squeeze else rhs)
    if b.dim() != 3 or tuple(b.shape[1:]) != (g.H, g.W):
        raise ValueError(f"rhs must be [n, {g.H}, {g.W}]")
    if not b.is_cuda:
        raise ValueError("rhs must be a CUDA tensor (no CPU path)")
    b = b.to(torch.complex128).contiguous()
    n_fields = b.shape[0]
    if initial is None:
        x = torch.zeros_like(b)
    else:
        x = torch.as_tensor(initial).to(b.device, torch.complex128).reshape(b.shape).clone().contiguous()
    lib = _lib.load()
    nbytes = lib.nsr_dense_solve_workspace_size(ctypes.byref(g.struct), n_fields, int(restart))
    if nbytes == 0:
        raise ValueError("unsupported dense grid for the preconditioner's transforms, or a bad restart length")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=b.device)
    per_field = torch.empty(n_fields, dtype=torch.float64, device=b.device)
    params = _lib.NsrDenseSolveParams(float(tolerance), float(shift), float((system.k0 * g.dx) ** 2),
                                      float(system.scal.real), float(system.scal.imag), int(restart),
                                      int(max_cycles), int(bool(adjoint)), 0)
    info = _lib.NsrDenseSolveInfo()
    _lib.check(lib.nsr_dense_solve(ctypes.byref(g.struct), ctypes.c_void_p(system.coef.data_ptr()),
                                   ctypes.byref(params), n_fields, ctypes.c_void_p(b.data_ptr()),
                                   ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(per_field.data_ptr()),
                                   ctypes.byref(info), ctypes.c_void_p(ws.data_ptr()), nbytes,
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    reason = _lib.REASONS[int(info.status)]
    if reason == "nonfinite":
        reason = "iteration_budget"   # the reference's GMRES knows only these two reasons
    x = x.to(rhs.dtype) if rhs.dtype in (torch.complex64, torch.complex128) else x
    return (x[0] if squeeze else x), {
        "reason": reason, "steps": int(info.steps), "residual": float(info.residual),
        "max_angle_residual": float(per_field.max()), "seconds": time.perf_counter() - started,
        "dtype": "complex64 Krylov / FP64 residual", "method": "gmres", "cycles": int(info.cycles)}


def homogeneous_reference(geometry: DenseGeometry, frequencies, lines, tolerance=1e-4, device="cuda"):
    """Reference pressure fields of the uniform medium (scripts/prepare_wave_teachers.py:22-35):
    for every frequency and source line ``lines [n_freq, n_angles, w]``, GMRES(32)
    on the uniform system with its own source.  Returns native fields
    complex64 ``[n_angles, n_freq, h, w]``, the layout of the on-disk
    ``reference/a{angle:02d}.npy`` arrays (nsrno/dense_wave.py:39-41)."""
    g = geometry
    lines = torch.as_tensor(lines, device=device)
    n_freq, n_angles = lines.shape[:2]
    out = torch.empty((n_angles, n_freq, g.h, g.w), dtype=torch.complex64, device=device)
    for k, f in enumerate(frequencies):
        s0 = homogeneous_system(g, f, device=device)
        src = s0.source(lines[k].to(torch.complex128))
        p, info = solve(s0, src, tolerance=tolerance, restart=32, max_cycles=80)
        if info["reason"] != "converged":
            raise RuntimeError(f"Homogeneous reference failed at {f} Hz: {info}")
        out[:, k] = p[:, g.pz:g.pz + g.h, g.px:g.px + g.w].to(torch.complex64)
    return out


def save_reference(directory, fields):
    """Write ``reference/a{angle:02d}.npy`` ([n_freq, h, w] complex64 each)."""
    from pathlib import Path
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    for a in range(fields.shape[0]):
        np.save(d / f"a{a:02d}.npy", fields[a].cpu().numpy())


# ---------------------------------------------------------------------------
# Implicit gradient and the converged, differentiable channels of the dense
# path (nsrno/dense_wave.py:227-259, nsrno/dense_surrogate.py:19-28).
# ---------------------------------------------------------------------------
def material_gradient(system: DenseSystem, medium, alpha, u_total, lam, line):
    """d/d(medium) of ``-Re sum conj(lam) mask [A(m)(mask u_total) - S(m) line]``,
    the scalar ImplicitChannels.backward differentiates (nsrno/dense_wave.py:250-255).

    The operator part goes through ``nsr_dense_grad`` (cotangents of the face
    coefficients and of the mass term, a contraction of the forward and adjoint
    fields on the device); the chain rule from those planes, and the source
    term, back to ``medium [2, h, w] = (c, rho)`` is torch autograd of
    :func:`medium_terms` (elementwise work on single planes)."""
    g = system.g
    lib = _lib.load()
    dev = system.coef.device
    u_total = torch.as_tensor(u_total).to(dev, torch.complex128).contiguous()
    lam = torch.as_tensor(lam).to(dev, torch.complex128).contiguous()
    if u_total.dim() == 2:
        u_total, lam = u_total[None], lam[None]
    n = u_total.shape[0]
    g_ax = torch.empty((g.H, g.W), dtype=torch.float64, device=dev)
    g_az = torch.empty_like(g_ax)
    g_mass = torch.empty((2, g.H, g.W), dtype=torch.float64, device=dev)
    _lib.check(lib.nsr_dense_grad(ctypes.byref(g.struct), ctypes.c_void_p(system.coef.data_ptr()),
                                  float(system.scal.real), float(system.scal.imag), n,
                                  ctypes.c_void_p(u_total.data_ptr()), ctypes.c_void_p(lam.data_ptr()),
                                  ctypes.c_void_p(g_ax.data_ptr()), ctypes.c_void_p(g_az.data_ptr()),
                                  ctypes.c_void_p(g_mass.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    with torch.enable_grad():
        m = torch.as_tensor(medium).detach().to(dev, torch.float64).requires_grad_(True)
        al = torch.as_tensor(alpha).detach().to(dev, torch.float64)
        t = medium_terms(g, m, al, system.frequency)
        surrogate = ((t["ax"] * g_ax).sum() + (t["az"] * g_az).sum() + (t["mass"].real * g_mass[0]).sum() +
                     (t["mass"].imag * g_mass[1]).sum())
        line = torch.as_tensor(line).to(dev)
        src = source_term(g, t, line.reshape(n, -1).to(torch.complex128))
        surrogate = surrogate + (lam.conj() * t["mask"] * src).real.sum()
        return torch.autograd.grad(surrogate, m)[0]


class DenseAcquisition:
    """The ``data`` of the dense path (the role of nsrno/dense_wave.py:15-57's
    DenseData): geometry, the source line of every (bin, angle), and the
    homogeneous-medium reference field of every (bin, angle), computed on
    first use by :func:`homogeneous_reference` and cached (the reference
    reads them from ``reference/a{angle:02d}.npy``)."""

    def __init__(self, geometry: DenseGeometry, bins, lines, references=None, device="cuda", tolerance=1e-8):
        self.geometry = geometry
        self.bins = [int(b) for b in bins]
        self.lines = torch.as_tensor(lines).to(device, torch.complex128)   # [bins, angles, w]
        self.device = torch.device(device)
        self.tolerance = tolerance
        self._refs = {}
        if references is not None:     # [angles, bins, h, w], the on-disk layout
            refs = torch.as_tensor(references)
            for k, b in enumerate(self.bins):
                self._refs[b] = g_pad(geometry, refs[:, k].to(self.device, torch.complex128))

    @staticmethod
    def frequency(frequency_bin):
        return frequency_bin * 40e6 / 2401

    def line(self, frequency_bin, angles):
        return self.lines[self.bins.index(frequency_bin)][list(angles)]

    def reference(self, frequency_bin, angles):
        if frequency_bin not in self._refs:
            lines = self.lines[self.bins.index(frequency_bin)][None]
            fields = homogeneous_reference(self.geometry, [self.frequency(frequency_bin)], lines,
                                           tolerance=self.tolerance, device=self.device)
            self._refs[frequency_bin] = g_pad(self.geometry, fields[:, 0].to(torch.complex128))
        return self._refs[frequency_bin][list(angles)]


def g_pad(geometry, native):
    """Native fields ``[n, h, w]`` on the padded grid."""
    return geometry.pad_field(native)


class DenseImplicitChannels(torch.autograd.Function):
    """Converged channels of the dense operator with the implicit adjoint gradient
    (ImplicitChannels, nsrno/dense_wave.py:227-256): the forward solves the
    scattered field of the assembled right-hand side (homogeneous-reference
    subtraction), the backward one adjoint solve and :func:`material_gradient`."""

    @staticmethod
    def forward(ctx, medium, alpha, data, frequency_bin, angles, tolerance):
        from .solver import receiver_response
        g = data.geometry
        f = data.frequency(frequency_bin)
        system = DenseSystem(g, medium.detach(), alpha.detach(), f, device=data.device)
        reference = homogeneous_system(g, f, device=data.device)
        line = data.line(frequency_bin, angles)
        pref = data.reference(frequency_bin, angles)
        rhs = assemble(system, reference, line, pref)
        u, info = solve(system, rhs, tolerance=tolerance)
        if info["reason"] != "converged":
            raise RuntimeError("Forward failed to converge: " + str(info))
        ctx.system, ctx.line, ctx.tolerance = system, line, tolerance
        ctx.save_for_backward(medium, alpha, u, pref)
        resp = receiver_response(f)
        return (u[:, g.face, torch.as_tensor(g.rx_cols, device=u.device)] * resp).to(torch.complex128)

    @staticmethod
    def backward(ctx, gradient):
        from .solver import receiver_response
        medium, alpha, u, pref = ctx.saved_tensors
        system = ctx.system
        g = system.g
        with torch.no_grad():
            rhs = torch.zeros_like(u)
            rhs[:, g.face, torch.as_tensor(g.rx_cols, device=u.device)] = \
                (gradient * receiver_response(system.frequency)).to(rhs.dtype)
            lam, info = solve(system, rhs, adjoint=True, tolerance=ctx.tolerance)
            if info["reason"] != "converged":
                raise RuntimeError("Adjoint failed to converge: " + str(info))
        derivative = material_gradient(system, medium, alpha, u + pref, lam, ctx.line)
        return derivative.to(medium.dtype), None, None, None, None, None


def dense_implicit_channels(medium, alpha, data: DenseAcquisition, frequency_bin, angles, tolerance=1e-5):
    """Differentiable converged receiver channels ``[A, 192]`` of the dense operator."""
    return DenseImplicitChannels.apply(medium, alpha, data, frequency_bin, list(angles), tolerance)


class DenseSurrogate(torch.nn.Module):
    """Drop-in for ``DenseSurrogate.forward`` (nsrno/dense_surrogate.py:19-28) on the
    8th-order dense operator: native ``medium [2, h, w]`` and ``alpha`` -> channels
    ``[A, 192]``, differentiable through the implicit adjoint."""

    def __init__(self, data: DenseAcquisition):
        super().__init__()
        self.data = data

    def forward(self, medium, alpha, frequency_bin, angles=None, tolerance=1e-5):
        if frequency_bin not in self.data.bins:
            raise ValueError("Frequency outside cached dense band")
        angles = list(range(self.data.lines.shape[1])) if angles is None else list(angles)
        return dense_implicit_channels(medium, alpha, self.data, frequency_bin, angles, tolerance)
