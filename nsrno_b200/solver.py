"""Record-level host API over the CUDA library.

Everything here runs on a CUDA device and goes through ``libnsrno_b200.so``;
there is no CPU path.  Tensors are PyTorch tensors on the current device and
kernels run on ``torch.cuda.current_stream()``.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from functools import lru_cache

import numpy as np
import torch

from . import _lib

DEFAULT_SHIFT = 0.15          # shifted-Laplace shift of nsrno/dense_wave.py:194
DEFAULT_REPLACE = 40          # true-residual period of nsrno/dense_wave.py:143
DEFAULT_RESTART = 1e-2        # restart BiCGSTAB after a 100x true-residual reduction


def _require_cuda(t: torch.Tensor, name: str):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (nsrno_b200 has no CPU path)")


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


@dataclass
class Geometry:
    """Grid, PML and array geometry of one record (lengths in metres)."""

    nz: int
    nx: int
    h: float
    n_pml: int
    face: int
    rx_cols: np.ndarray
    aperture_half_width: float
    c0: float = 1500.0
    rho0: float = 1000.0
    pml_strength: float = 12.0
    alpha_power: float = 1.1

    @classmethod
    def from_record(cls, rec):
        return cls(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, face=rec.face,
                   rx_cols=np.asarray(rec.rx_cols), aperture_half_width=rec.aperture_half_width,
                   c0=rec.c0, rho0=rec.rho0, pml_strength=rec.pml_strength, alpha_power=rec.alpha_power)

    @property
    def n(self):
        return self.nz * self.nx

    def struct(self):
        return _lib.NsrGrid(self.nz, self.nx, self.n_pml, self.face, self.h, self.c0, self.rho0,
                            self.pml_strength, self.alpha_power, self.aperture_half_width)

    def rx_index(self, device):
        flat = self.face * self.nx + np.asarray(self.rx_cols, dtype=np.int64)
        return torch.as_tensor(flat.astype(np.int32), device=device)


class Medium:
    """Material planes (a, b, t) of one record resident in device memory."""

    def __init__(self, geometry: Geometry, c, rho, alpha, device=None):
        device = torch.device(device or "cuda")
        self.geometry = geometry
        shape = (geometry.nz, geometry.nx)
        planes = []
        for name, v in (("c", c), ("rho", rho), ("alpha", alpha)):
            t = torch.as_tensor(v, dtype=torch.float32).to(device)
            if tuple(t.shape) != shape:
                raise ValueError(f"{name} must have shape {shape}")
            planes.append(t.contiguous())
        self.c, self.rho, self.alpha = planes
        if not bool(torch.isfinite(self.c).all() and (self.c > 0).all() and
                    torch.isfinite(self.rho).all() and (self.rho > 0).all() and torch.isfinite(self.alpha).all()):
            raise ValueError("c and rho must be finite and positive; alpha must be finite")
        _require_cuda(self.c, "medium")
        self._grid = geometry.struct()
        lib = _lib.load()
        nbytes = lib.nsr_material_bytes(ctypes.byref(self._grid))
        if nbytes == 0:
            raise ValueError("invalid grid")
        self.material = torch.empty(nbytes, dtype=torch.uint8, device=device)
        _lib.check(lib.nsr_setup_material(ctypes.byref(self._grid), _ptr(self.c), _ptr(self.rho),
                                          _ptr(self.alpha), _ptr(self.material), _stream()))

    @property
    def device(self):
        return self.material.device

    @property
    def coef(self):
        """Float planes (a, b, t) ``[3, nz, nx]`` used by the FP32 Krylov kernels."""
        g = self.geometry
        return self.material[: 12 * g.n].view(torch.float32).view(3, g.nz, g.nx)

    @property
    def coef64(self):
        """Double planes (a, b, t) ``[3, nz, nx]`` used by the FP64 residual, apply and gradient."""
        g = self.geometry
        off = (12 * g.n + 255) // 256 * 256
        return self.material[off: off + 24 * g.n].view(torch.float64).view(3, g.nz, g.nx)


@dataclass
class BatchResult:
    iq: torch.Tensor            # complex128 [S, n_rx]
    residual: torch.Tensor      # float64 [S] true relative residual
    iterations: torch.Tensor    # int32 [S]
    status: torch.Tensor        # int32 [S]
    fields: torch.Tensor | None = None   # complex64 [S, nz, nx]
    seconds: float = 0.0
    extra: dict = field(default_factory=dict)

    def reasons(self):
        return [_lib.REASONS[int(s)] for s in self.status.cpu()]


class Workspace:
    """Reusable device workspace for ``solve_batched`` (grows on demand)."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes, device):
        if self.buf is None or self.buf.numel() < nbytes or self.buf.device != device:
            self.buf = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        return self.buf


_default_ws = Workspace()


def solve_batched(medium: Medium, freqs, angles=None, *, rhs=None, x0=None, tolerance=1e-6,
                  max_iterations=2000, shift=DEFAULT_SHIFT, replace_every=DEFAULT_REPLACE, n_slots=16,
                  adjoint=False, return_fields=False, rx_index=None, graph_iterations=16,
                  profile_iterations=0, restart_factor=DEFAULT_RESTART, warm_gate=1.0, fields_dtype=torch.complex64,
                  learned=None, gain_index=None, time_limit=0.0, tiles=None, blocking=None,
                  workspace: Workspace | None = None, out: BatchResult | None = None) -> BatchResult:
    """Solve every (frequency, angle) system of a record with batched BiCGSTAB.

    ``freqs``/``angles`` are 1-D (one entry per system).  ``rhs`` (complex64
    [S, nz, nx], SI units) replaces the plane-wave source when given.
    ``x0`` (complex64 [S, nz, nx]) is a warm start.  ``learned`` (a
    :class:`nsrno_b200.learned.LearnedSetup`) replaces the fixed preconditioner
    by the learned one; ``gain_index`` (int [S]) picks each system's gain pair
    (default: its position in ``learned.freqs``).  ``time_limit`` (seconds,
    0: none) bounds each system's solve on the device: a system still running
    then stops at its next true residual with reason ``"timeout"``.
    ``tiles`` (a dict of :class:`nsrno_b200._lib.NsrTiles` fields, e.g. from
    :func:`nsrno_b200.tune.tuned_config`) overrides the launch shapes.
    ``blocking`` (default: only when ``profile_iterations`` > 0) selects the
    host-polled ``nsr_solve_batched_sync``, which also reports the device loop
    time and per-kernel timings in ``extra["stats"]``; otherwise the solve is
    one device-side graph loop enqueued on the current stream
    (``nsr_solve_batched``) and this call returns before it finishes.
    """
    lib = _lib.load()
    g = medium.geometry
    dev = medium.device
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    S = int(freqs.numel())
    if angles is None and rhs is None:
        raise ValueError("either angles (plane-wave sources) or rhs must be given")
    if angles is not None:
        angles = torch.as_tensor(angles, dtype=torch.float64, device=dev).reshape(-1).contiguous()
        if angles.numel() != S:
            raise ValueError("freqs and angles must have the same length")
    def field_arg(t, name):
        if t is None:
            return None
        t = torch.as_tensor(t)
        if tuple(t.shape) != (S, g.nz, g.nx) or not t.is_complex():
            raise ValueError(f"{name} must be a complex tensor of shape {(S, g.nz, g.nx)}")
        return t.to(dev, torch.complex64).contiguous()

    rhs = field_arg(rhs, "rhs")
    x0 = field_arg(x0, "x0")
    if rx_index is None:
        rx_index = g.rx_index(dev)
    n_rx = int(rx_index.numel())
    n_slots = max(1, min(int(n_slots), S)) if S else 1
    grid = medium._grid
    ws_bytes = lib.nsr_solve_workspace_size(ctypes.byref(grid), n_slots)
    if ws_bytes == 0:
        raise ValueError("unsupported grid for the batched solver (nz, nx in [8, 2048] with no prime factor above 61)")
    ws = (workspace or _default_ws).get(ws_bytes, dev)
    if out is None:
        out = BatchResult(iq=torch.empty((S, n_rx), dtype=torch.complex128, device=dev),
                          residual=torch.empty(S, dtype=torch.float64, device=dev),
                          iterations=torch.empty(S, dtype=torch.int32, device=dev),
                          status=torch.empty(S, dtype=torch.int32, device=dev),
                          fields=torch.empty((S, g.nz, g.nx), dtype=fields_dtype, device=dev)
                          if return_fields else None)
    if fields_dtype not in (torch.complex64, torch.complex128):
        raise ValueError("fields_dtype must be complex64 or complex128")
    if out.fields is not None and (out.fields.dtype != fields_dtype or tuple(out.fields.shape) != (S, g.nz, g.nx)):
        raise ValueError("out.fields does not match fields_dtype and the system count")
    params = _lib.NsrSolveParams(float(tolerance), float(shift), float(restart_factor), float(warm_gate),
                                 int(max_iterations),
                                 int(replace_every),
                                 int(n_slots), int(bool(adjoint)), int(graph_iterations), int(profile_iterations),
                                 int(fields_dtype == torch.complex128), 0)
    keep = _learned_params(params, learned, gain_index, freqs)
    if not time_limit >= 0.0:
        raise ValueError("time_limit must be >= 0")
    params.time_limit_s = float(time_limit)
    tiles_struct = _tiles_struct(tiles)
    if tiles_struct is not None:
        params.tiles = ctypes.pointer(tiles_struct)
    stats = _lib.NsrSolveStats()
    if blocking is None:
        blocking = profile_iterations > 0
    entry = lib.nsr_solve_batched_sync if blocking else lib.nsr_solve_batched
    _lib.check(entry(
        ctypes.byref(grid), _ptr(medium.material), _ptr(freqs), _ptr(angles), S,
        _ptr(rhs), _ptr(x0), _ptr(rx_index), n_rx, ctypes.byref(params),
        _ptr(ws), ws.numel(), _ptr(out.iq), _ptr(out.residual), _ptr(out.iterations), _ptr(out.status),
        _ptr(out.fields), ctypes.byref(stats), _stream()))
    del keep, tiles_struct
    out.extra["stats"] = stats.as_dict()
    out.extra["blocking"] = bool(blocking)
    out.extra["n_slots"] = n_slots
    if not blocking:
        out.extra["stats"]["loop_ms"] = None
        # the progress record (finished systems, device loop rounds, error),
        # copied to pinned memory behind the solve; read it after a sync
        off = lib.nsr_solve_progress_offset(ctypes.byref(grid), n_slots)
        words = torch.empty(8, dtype=torch.int32, pin_memory=True)
        words.copy_(ws[off:off + 32].view(torch.int32), non_blocking=True)
        groups = int((tiles or {}).get("slot_groups", 0)) or (2 if n_slots >= 8 else 1)
        per_round = 9 * int(graph_iterations) * min(groups, n_slots) + 1
        out.extra["progress_words"] = words
        out.extra["launches_per_round"] = per_round
    return out


def solve_progress(result: BatchResult):
    """(systems finished, device loop rounds, error flag, kernels launched) of a
    non-blocking solve, from the progress record copied behind it (call after
    the stream has passed the solve, e.g. after torch.cuda.synchronize()).
    For a blocking solve the host already counted everything: (systems,
    graph launches, 0, kernels launched)."""
    if result.extra.get("blocking"):
        st = result.extra["stats"]
        return int(result.status.numel()), int(st.get("graph_launches", 0)), 0, int(st["launches"])
    w = result.extra["progress_words"]
    rounds = int(w[6:8].view(torch.int64)[0])
    launches = result.extra["stats"]["launches"] + rounds * result.extra["launches_per_round"]
    return int(w[1]), rounds, int(w[4]), launches


def _tiles_struct(tiles):
    """NsrTiles from a dict of its fields (None: built-in launch shapes)."""
    if tiles is None:
        return None
    if isinstance(tiles, _lib.NsrTiles):
        return tiles
    unknown = set(tiles) - set(_lib.NsrTiles.FIELDS)
    if unknown:
        raise ValueError(f"unknown tile fields {sorted(unknown)}")
    t = _lib.NsrTiles()
    for k, v in tiles.items():
        setattr(t, k, int(v))
    return t


def _learned_params(params, learned, gain_index, freqs):
    """Attach the learned preconditioner to solver parameters; returns what must stay alive."""
    if learned is None:
        return None
    if gain_index is None:
        gain_index = learned.index_of(freqs)
    gain_index = torch.as_tensor(gain_index, dtype=torch.int32, device=freqs.device).reshape(-1).contiguous()
    if gain_index.numel() != freqs.numel():
        raise ValueError("gain_index needs one entry per system")
    struct = learned.struct(gain_index)
    params.learned = ctypes.pointer(struct)
    return (struct, gain_index)


def gmres_batched(medium: Medium, freqs, angles=None, *, rhs=None, x0=None, tolerance=1e-6, max_iterations=2560,
                  restart=32, shift=DEFAULT_SHIFT, n_slots=16, adjoint=False, return_fields=False,
                  fields_dtype=torch.complex64, rx_index=None, learned=None, gain_index=None,
                  workspace: Workspace | None = None) -> BatchResult:
    """Restarted GMRES(restart) for every system (nsrno/wave_solver.py:9-36 on the device).

    Same inputs and outputs as :func:`solve_batched`; ``iterations`` counts
    Arnoldi steps, i.e. operator applications.
    """
    lib = _lib.load()
    g = medium.geometry
    dev = medium.device
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    S = int(freqs.numel())
    if angles is None and rhs is None:
        raise ValueError("either angles (plane-wave sources) or rhs must be given")
    if angles is not None:
        angles = torch.as_tensor(angles, dtype=torch.float64, device=dev).reshape(-1).contiguous()
        if angles.numel() != S:
            raise ValueError("freqs and angles must have the same length")

    def field_arg(t, name):
        if t is None:
            return None
        t = torch.as_tensor(t)
        if tuple(t.shape) != (S, g.nz, g.nx) or not t.is_complex():
            raise ValueError(f"{name} must be a complex tensor of shape {(S, g.nz, g.nx)}")
        return t.to(dev, torch.complex64).contiguous()

    rhs = field_arg(rhs, "rhs")
    x0 = field_arg(x0, "x0")
    if rx_index is None:
        rx_index = g.rx_index(dev)
    n_rx = int(rx_index.numel())
    n_slots = max(1, min(int(n_slots), S)) if S else 1
    grid = medium._grid
    ws_bytes = lib.nsr_gmres_workspace_size(ctypes.byref(grid), n_slots, int(restart))
    if ws_bytes == 0:
        raise ValueError("unsupported grid or restart length for GMRES")
    ws = (workspace or _default_ws).get(ws_bytes, dev)
    out = BatchResult(iq=torch.empty((S, n_rx), dtype=torch.complex128, device=dev),
                      residual=torch.empty(S, dtype=torch.float64, device=dev),
                      iterations=torch.empty(S, dtype=torch.int32, device=dev),
                      status=torch.empty(S, dtype=torch.int32, device=dev),
                      fields=torch.empty((S, g.nz, g.nx), dtype=fields_dtype, device=dev) if return_fields else None)
    params = _lib.NsrGmresParams(float(tolerance), float(shift), int(max_iterations), int(restart), int(n_slots),
                                 int(bool(adjoint)), int(fields_dtype == torch.complex128), 0)
    keep = _learned_params(params, learned, gain_index, freqs)  # noqa: F841 (kept alive for the call)
    _lib.check(lib.nsr_gmres_batched(
        ctypes.byref(grid), _ptr(medium.material), _ptr(freqs), _ptr(angles), S, _ptr(rhs), _ptr(x0),
        _ptr(rx_index), n_rx, ctypes.byref(params), _ptr(ws), ws.numel(), _ptr(out.iq), _ptr(out.residual),
        _ptr(out.iterations), _ptr(out.status), _ptr(out.fields), _stream()))
    return out


def apply(medium: Medium, x: torch.Tensor, freqs, adjoint=False):
    """``A x`` (or ``A^H x``) of the h^2-scaled operator for fields x [S, nz, nx]."""
    g = medium.geometry
    _require_cuda(x, "x")
    if x.dtype not in (torch.complex64, torch.complex128) or x.dim() != 3 or tuple(x.shape[1:]) != (g.nz, g.nx):
        raise ValueError("x must be complex64/complex128 [S, nz, nx]")
    x = x.contiguous()
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=x.device).reshape(-1).contiguous()
    if freqs.numel() != x.shape[0]:
        raise ValueError("one frequency per field")
    y = torch.empty_like(x)
    _lib.check(_lib.load().nsr_apply(ctypes.byref(medium._grid), _ptr(medium.material), _ptr(freqs), x.shape[0],
                                     int(bool(adjoint)), 0 if x.dtype == torch.complex64 else 1,
                                     _ptr(x), _ptr(y), _stream()))
    return y


def precondition(medium: Medium, x: torch.Tensor, freqs, shift=DEFAULT_SHIFT, adjoint=False):
    """``M^-1 x`` of the FFT shifted-Laplace preconditioner, x complex64 [S, nz, nx]."""
    g = medium.geometry
    _require_cuda(x, "x")
    if x.dtype != torch.complex64 or x.dim() != 3 or tuple(x.shape[1:]) != (g.nz, g.nx):
        raise ValueError("x must be complex64 [S, nz, nx]")
    x = x.contiguous()
    S = x.shape[0]
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=x.device).reshape(-1).contiguous()
    lib = _lib.load()
    nbytes = lib.nsr_precondition_workspace_size(ctypes.byref(medium._grid), S)
    if nbytes == 0:
        raise ValueError("unsupported grid for the preconditioner")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
    y = torch.empty_like(x)
    _lib.check(lib.nsr_precondition(ctypes.byref(medium._grid), _ptr(freqs), S, float(shift), int(bool(adjoint)),
                                    _ptr(x), _ptr(y), _ptr(ws), nbytes, _stream()))
    return y


def plane_wave_rhs(medium: Medium, freqs, angles):
    """SI right-hand sides ``-line/h^2`` on the array row, complex128 [S, nz, nx]."""
    g = medium.geometry
    dev = medium.device
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    angles = torch.as_tensor(angles, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    b = torch.empty((freqs.numel(), g.nz, g.nx), dtype=torch.complex128, device=dev)
    _lib.check(_lib.load().nsr_plane_wave_rhs(ctypes.byref(medium._grid), _ptr(freqs), _ptr(angles),
                                              freqs.numel(), _ptr(b), _stream()))
    return b


def grad_accum(medium: Medium, freqs, u: torch.Tensor, lam: torch.Tensor, g_logc=None, g_logrho=None):
    """Accumulate ``-Re(lam^H dA/dm u)`` over systems for m = log c, log rho (float64 planes)."""
    g = medium.geometry
    dev = medium.device
    for name, t in (("u", u), ("lam", lam)):
        _require_cuda(t, name)
        if t.dtype not in (torch.complex64, torch.complex128) or t.dim() != 3 or tuple(t.shape[1:]) != (g.nz, g.nx):
            raise ValueError(f"{name} must be complex64 or complex128 [S, nz, nx]")
    dtype = torch.complex128 if torch.complex128 in (u.dtype, lam.dtype) else torch.complex64
    u = u.to(dtype).contiguous()
    lam = lam.to(dtype).contiguous()
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    if g_logc is None:
        g_logc = torch.zeros((g.nz, g.nx), dtype=torch.float64, device=dev)
    if g_logrho is None:
        g_logrho = torch.zeros((g.nz, g.nx), dtype=torch.float64, device=dev)
    _lib.check(_lib.load().nsr_grad_accum(ctypes.byref(medium._grid), _ptr(medium.material), _ptr(freqs), u.shape[0],
                                          int(dtype == torch.complex128), _ptr(u), _ptr(lam), _ptr(g_logc),
                                          _ptr(g_logrho), _stream()))
    return g_logc, g_logrho


@lru_cache(maxsize=512)
def receiver_response(frequency, dt=2.5e-9):
    """Known receive-chain transfer at one frequency (nsrno/conditioned_data.py:10-24).

    4th-order Butterworth band-pass 4-7.5 MHz applied forward and backward
    (|H|^2) times the real part of the linear-phase-corrected Kaiser FIR of the
    10x polyphase decimation.  A real scalar.
    """
    from scipy.signal import butter, firwin, freqz, sosfreqz

    sos = butter(4, [4e6, 7.5e6], fs=1 / dt, btype="bandpass", output="sos")
    _, h = sosfreqz(sos, worN=[frequency], fs=1 / dt)
    down = 10
    half_len = 10 * down
    taps = firwin(2 * half_len + 1, 1 / down, window=("kaiser", 5.0))
    omega = 2 * np.pi * frequency * dt
    _, fir = freqz(taps, worN=[omega])
    return float(abs(h[0]) ** 2 * (fir[0] * np.exp(1j * omega * half_len)).real)


def band_rf(spectrum, bins, n_samples=2401):
    """Band-limited RF traces ``[n_channels, n_samples]`` (float64) from receiver
    spectra ``[n_channels, n_bins]`` on positive bins (predict_band_rf,
    nsrno/wave_operator.py:169-180: ``irfft`` with 'forward' normalisation of a
    spectrum that is zero elsewhere).  Raises ``ValueError('Positive RF bin out
    of range')`` like the reference."""
    spectrum = torch.as_tensor(spectrum)
    _require_cuda(spectrum, "spectrum")
    bins_np = np.asarray(bins, dtype=np.int64).reshape(-1)
    if spectrum.dim() != 2 or spectrum.shape[1] != bins_np.size:
        raise ValueError("spectrum must be [n_channels, n_bins]")
    if ((bins_np <= 0) | (2 * bins_np >= n_samples)).any():
        raise ValueError("Positive RF bin out of range")
    spec = spectrum.to(torch.complex128).contiguous()
    b = torch.as_tensor(bins_np.astype(np.int32), device=spec.device)
    out = torch.empty((spec.shape[0], int(n_samples)), dtype=torch.float64, device=spec.device)
    _lib.check(_lib.load().nsr_band_rf(spec.shape[0], int(bins_np.size), int(n_samples), _ptr(spec), _ptr(b),
                                       _ptr(out), _stream()))
    return out


def receiver_rf(iq, frequency_bins, response=True, n_samples=2401, clock_hz=40e6):
    """RF traces of the receiver IQ of a record's bins: ``iq [n_bins, n_channels]``
    times the receive response of each bin (nsrno/conditioned_data.py:10-24),
    then :func:`band_rf`."""
    iq = torch.as_tensor(iq)
    bins = np.asarray(frequency_bins, dtype=np.int64).reshape(-1)
    if response:
        r = torch.as_tensor([receiver_response(float(k) * clock_hz / n_samples) for k in bins],
                            dtype=torch.float64, device=iq.device)
        iq = iq.to(torch.complex128) * r[:, None]
    return band_rf(iq.transpose(0, 1), bins, n_samples)


def true_residual(medium: Medium, x: torch.Tensor, freqs, angles=None, rhs=None, adjoint=False):
    """FP64 true relative residuals ``||b - A x|| / ||b||`` [S] of fields x [S, nz, nx]
    (``nsr_true_residual``); ``b`` is ``rhs`` (SI) or the plane-wave source of (freqs, angles)."""
    g = medium.geometry
    _require_cuda(x, "x")
    if x.dim() != 3 or tuple(x.shape[1:]) != (g.nz, g.nx) or not x.is_complex():
        raise ValueError("x must be complex [S, nz, nx]")
    dev = x.device
    x = x.to(torch.complex128).contiguous()
    S = x.shape[0]
    freqs = torch.as_tensor(freqs, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    if rhs is None and angles is None:
        raise ValueError("either angles or rhs must be given")
    ang = None if angles is None else torch.as_tensor(angles, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    b = None if rhs is None else torch.as_tensor(rhs).to(dev, torch.complex128).contiguous()
    lib = _lib.load()
    nbytes = lib.nsr_true_residual_workspace_size(ctypes.byref(medium._grid), S)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = torch.empty(S, dtype=torch.float64, device=dev)
    _lib.check(lib.nsr_true_residual(ctypes.byref(medium._grid), _ptr(medium.material), _ptr(freqs), _ptr(ang), S,
                                     int(bool(adjoint)), _ptr(x), _ptr(b), _ptr(out), _ptr(ws), nbytes, _stream()))
    return out
