"""CPU oracle for the 5-point viscoacoustic Helmholtz solve -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only to check results or as the timed
CPU baseline.  The product path (``nsrno_b200``) never imports it.

It restates, in complex128 NumPy/SciPy, the discretisation of the reference
``nsrno/theranostic/wave.py``:

* ``Solver._stretch``        theranostic/wave.py:127-135  -> :func:`stretch`
* ``Solver.coefficients``    theranostic/wave.py:137-156  -> :func:`edge_weights`
* ``Solver.matrix``          theranostic/wave.py:174-188  -> :func:`operator`
* ``Solver.solve``           theranostic/wave.py:240-273  -> :func:`solve_lu`
* ``Solver.born_jacobian``   theranostic/wave.py:331-389  -> :func:`material_gradient`
  (the same exact derivative, contracted with an adjoint field instead of
  being formed column by column)

and the Krylov drivers of the dense path:

* ``bicgstab``   nsrno/dense_wave.py:118-148  -> :func:`bicgstab`
* ``gmres``      nsrno/wave_solver.py:9-36    -> :func:`gmres`

Two extensions follow the solve contract (c, rho, alpha, freq, angle, source)
and are stated here because the
5-point reference has no counterpart for them:

* power-law attenuation folded into the mass term, ``k^2 -> k^2 (1 + i e)^2``
  with ``e = alpha_Np(f) c / omega``; nsrno/wave_operator.py:56,67 writes the
  same factor as ``(1 - i alpha c / omega)^2`` in its opposite time
  convention.  With the ``exp(-i omega t)`` convention and the ``1 + i sigma/omega``
  stretch of theranostic/wave.py the decaying sign is ``+i``;
* a steered plane-wave line source with the cosine aperture taper of
  nsrno/wave_operator.py:111-115, placed on one grid row.

Unknowns are ordered ``[z, x]`` row-major like the reference grid.  With
``a = rho0/rho`` (= 1 + m_eta) and ``b = rho0 c0^2 / (rho c^2)`` (= 1 + m_kappa)
the assembled equation is

    sum_edges  w_e (a_i + a_j)/(2 h^2) (p_j - p_i)  +  k0^2 sx sz b (1 + i e)^2 p_i  =  rhs_i

with the ghost value ``p = 0`` and ghost contrast zero (``a = 1``) outside the
grid, exactly the reference's zero-ghost boundary edges.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
from scipy import sparse
from scipy.sparse.linalg import splu

NEPER_PER_DB_CM = 100.0 * math.log(10.0) / 20.0  # dB/cm -> Np/m


@dataclass
class Spec:
    """Grid, PML and acquisition of one record (all lengths in metres)."""

    nz: int
    nx: int
    h: float
    n_pml: int
    c0: float = 1500.0
    rho0: float = 1000.0
    pml_strength: float = 12.0
    face: int = 0
    rx_cols: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    aperture_half_width: float = 0.0
    alpha_power: float = 1.1

    @property
    def n(self):
        return self.nz * self.nx

    def axes(self):
        """Node coordinates: x centred on the grid, z measured from row 0."""
        x = (np.arange(self.nx) - (self.nx - 1) / 2.0) * self.h
        z = np.arange(self.nz) * self.h
        return x, z


def stretch(coord, lower, upper, width, sigma_max, omega):
    """Quadratic complex stretch ``1 + i sigma(x)/omega`` (theranostic/wave.py:127-135)."""
    coord = np.asarray(coord, dtype=np.float64)
    if width == 0:
        return np.ones_like(coord, dtype=np.complex128)
    fraction = np.maximum((lower + width - coord) / width, (coord - upper + width) / width)
    profile = np.clip(fraction, 0.0, 1.0) ** 2
    return 1.0 + 1j * (sigma_max / omega) * profile


def stretches(spec: Spec, frequency_hz: float):
    """Node and half-node stretches.

    Returns ``(sx[nx], sz[nz], sxh[nx+1], szh[nz+1])``; the half-node arrays run
    from ``x[0]-h/2`` to ``x[-1]+h/2`` so that their first and last entries are
    the outer (ghost-edge) stretches of theranostic/wave.py:148-149.
    """
    omega = 2.0 * math.pi * frequency_hz
    x, z = spec.axes()
    width = spec.n_pml * spec.h
    sigma_max = spec.pml_strength * spec.c0 / width if width > 0 else 0.0
    xh = np.concatenate(([x[0] - spec.h / 2], (x[:-1] + x[1:]) / 2, [x[-1] + spec.h / 2]))
    zh = np.concatenate(([z[0] - spec.h / 2], (z[:-1] + z[1:]) / 2, [z[-1] + spec.h / 2]))
    sx = stretch(x, x[0], x[-1], width, sigma_max, omega)
    sz = stretch(z, z[0], z[-1], width, sigma_max, omega)
    sxh = stretch(xh, x[0], x[-1], width, sigma_max, omega)
    szh = stretch(zh, z[0], z[-1], width, sigma_max, omega)
    return sx, sz, sxh, szh


def material(spec: Spec, c, rho, alpha_db):
    """``(a, b, t)``: inverse density ratio, compressibility ratio, attenuation slope.

    ``t`` is defined so that ``e(f) = alpha_Np(f) c / omega = t (f/1MHz)^(y-1)``.
    """
    c = np.asarray(c, dtype=np.float64)
    rho = np.asarray(rho, dtype=np.float64)
    alpha_db = np.asarray(alpha_db, dtype=np.float64)
    a = spec.rho0 / rho
    b = spec.rho0 * spec.c0 ** 2 / (rho * c ** 2)
    t = alpha_db * NEPER_PER_DB_CM * c / (2.0 * math.pi * 1e6)
    return a, b, t


def k0_of(spec: Spec, frequency_hz: float):
    return 2.0 * math.pi * frequency_hz / spec.c0


def edge_weights(spec: Spec, a, frequency_hz: float):
    """Stretched edge fluxes ``Fx[nz, nx+1]`` and ``Fz[nz+1, nx]`` in SI.

    ``Fx[:, j]`` joins node ``j-1`` and node ``j`` (``j=0`` and ``j=nx`` are the
    ghost edges), likewise ``Fz`` along z.  Ghost contrast is zero, so the ghost
    side uses ``a = 1``.  Edge weights follow ``stretch * (1 + edge_average(m_eta))
    / h^2`` of theranostic/wave.py:150-155,179.
    """
    sx, sz, sxh, szh = stretches(spec, frequency_hz)
    ap = np.pad(np.asarray(a, dtype=np.float64), 1, constant_values=1.0)
    ax = 0.5 * (ap[1:-1, :-1] + ap[1:-1, 1:])      # [nz, nx+1]
    az = 0.5 * (ap[:-1, 1:-1] + ap[1:, 1:-1])      # [nz+1, nx]
    fx = (sz[:, None] / sxh[None, :]) * ax / spec.h ** 2
    fz = (sx[None, :] / szh[:, None]) * az / spec.h ** 2
    return fx, fz


def mass(spec: Spec, b, t, frequency_hz: float):
    """Stretched complex mass ``k0^2 sx sz b (1 + i e)^2`` (theranostic/wave.py:180 + attenuation)."""
    sx, sz, _, _ = stretches(spec, frequency_hz)
    e = np.asarray(t) * (frequency_hz / 1e6) ** (spec.alpha_power - 1.0)
    return k0_of(spec, frequency_hz) ** 2 * (sz[:, None] * sx[None, :]) * np.asarray(b) * (1.0 + 1j * e) ** 2


def operator(spec: Spec, c, rho, alpha_db, frequency_hz: float):
    """Assemble the complex-symmetric 5-point matrix (CSR, complex128, SI units)."""
    return operator_planes(spec, *material(spec, c, rho, alpha_db), frequency_hz)


def operator_planes(spec: Spec, a, b, t, frequency_hz: float):
    """The same matrix from the planes ``a = 1 + m_eta``, ``b = 1 + m_kappa`` and ``t``."""
    fx, fz = edge_weights(spec, a, frequency_hz)
    m = mass(spec, b, t, frequency_hz)
    diagonal = m - fx[:, :-1] - fx[:, 1:] - fz[:-1, :] - fz[1:, :]
    nz, nx = spec.nz, spec.nx
    east = fx[:, 1:-1]                       # edge (i,j)-(i,j+1), j < nx-1
    east_full = np.zeros((nz, nx), dtype=np.complex128)
    east_full[:, :-1] = east
    south = fz[1:-1, :].ravel()              # edge (i,j)-(i+1,j)
    e1 = east_full.ravel()[:-1]
    return sparse.diags(
        [diagonal.ravel(), e1, e1, south, south],
        [0, 1, -1, nx, -nx],
        shape=(spec.n, spec.n),
        format="csr",
        dtype=np.complex128,
    )


def plane_wave_line(spec: Spec, frequency_hz: float, angle_rad: float):
    """Steered line source on row ``face``: ``taper(x) exp(-i k0 x sin(theta))``.

    Aperture taper ``0.5 (1 + cos(pi x / X))`` for ``|x| <= X`` as in
    nsrno/wave_operator.py:114-115, with ``X`` the half-width of the array.
    """
    x, _ = spec.axes()
    half = spec.aperture_half_width
    taper = np.where(np.abs(x) <= half, 0.5 * (1.0 + np.cos(math.pi * x / half)), 0.0)
    return taper * np.exp(-1j * k0_of(spec, frequency_hz) * x * math.sin(angle_rad))


def plane_wave_rhs(spec: Spec, frequency_hz: float, angle_rad: float):
    """Right-hand side ``-W/h^2`` with unit nodal weights on the source row (theranostic/wave.py:260)."""
    rhs = np.zeros((spec.nz, spec.nx), dtype=np.complex128)
    rhs[spec.face] = -plane_wave_line(spec, frequency_hz, angle_rad) / spec.h ** 2
    return rhs.ravel()


def receivers(spec: Spec, fields):
    """Receiver IQ: nodal samples on the array row (nsrno/dense_wave.py:64)."""
    fields = np.asarray(fields)
    return fields.reshape(fields.shape[:-1] + (spec.nz, spec.nx))[..., spec.face, spec.rx_cols]


def solve_lu(matrix, rhs):
    """SuperLU direct solve (theranostic/wave.py:253-261). ``rhs`` is ``[n]`` or ``[n, k]``."""
    lu = splu(matrix.tocsc())
    return lu.solve(np.asarray(rhs, dtype=np.complex128))


def relative_residual(matrix, x, rhs):
    return float(np.linalg.norm(matrix @ x - rhs) / max(np.linalg.norm(rhs), 1e-300))


def bicgstab(apply, rhs, x=None, tolerance=1e-3, max_iterations=800, replace_every=40):
    """Unpreconditioned BiCGSTAB with the reference's decisions (dense_wave.py:118-148).

    Breakdown below 1e-30, true-residual replacement every ``replace_every``
    iterations, divergence above 1e5.  Returns ``(x, info)`` with the
    reference's ``reason``/``iterations``/``residual`` keys.
    """
    rhs = np.asarray(rhs, dtype=np.complex128)
    x = np.zeros_like(rhs) if x is None else np.array(x, dtype=np.complex128)
    scale = max(np.linalg.norm(rhs), 1e-30)
    r = rhs - apply(x)
    shadow = r.copy()
    p = np.zeros_like(r)
    v = np.zeros_like(r)
    rho_old = alpha = omega = 1.0 + 0j
    reason, used = "iteration_budget", 0
    for iteration in range(max_iterations):
        if np.linalg.norm(r) / scale < tolerance:
            reason = "converged"
            break
        rho = np.vdot(shadow, r)
        if not np.isfinite(rho) or abs(rho) < 1e-30 or abs(omega) < 1e-30:
            reason = "breakdown"
            break
        beta = (rho / rho_old) * (alpha / omega)
        p = r + beta * (p - omega * v)
        v = apply(p)
        denominator = np.vdot(shadow, v)
        if abs(denominator) < 1e-30:
            reason = "breakdown"
            break
        alpha = rho / denominator
        s = r - alpha * v
        if np.linalg.norm(s) / scale < tolerance:
            x = x + alpha * p
            r = s
            used = iteration + 1
            reason = "converged"
            break
        t = apply(s)
        omega = np.vdot(t, s) / max(np.vdot(t, t).real, 1e-30)
        x = x + alpha * p + omega * s
        r = s - omega * t
        rho_old = rho
        used = iteration + 1
        if replace_every and iteration % replace_every == replace_every - 1:
            r = rhs - apply(x)
            if not np.isfinite(r).all() or np.linalg.norm(r) / scale > 1e5:
                reason = "diverged"
                break
    actual = float(np.linalg.norm(apply(x) - rhs) / scale)
    if actual < tolerance:
        reason = "converged"
    return x, dict(reason=reason, iterations=used, residual=actual, method="BiCGSTAB")


def gmres(apply, rhs, x=None, restart=30, max_cycles=200, tolerance=1e-7, callback=None, precondition=None):
    """Restarted right-preconditioned GMRES with two classical Gram-Schmidt passes (wave_solver.py:9-36).

    ``precondition`` is the right preconditioner (identity when None); the
    preconditioned directions are kept as in the reference.  Happy breakdown
    below 1e-12; the small least-squares problem is solved in complex128 with
    ``lstsq`` as in the reference.  Returns ``(x, reason, steps)``.
    """
    rhs = np.asarray(rhs, dtype=np.complex128)
    x = np.zeros_like(rhs) if x is None else np.array(x, dtype=np.complex128)
    scale = max(np.linalg.norm(rhs), 1e-30)
    n = rhs.size
    basis = np.empty((restart + 1, n), dtype=np.complex128)
    directions = np.empty((restart, n), dtype=np.complex128)
    precondition = precondition or (lambda v: v)
    steps = 0
    for _ in range(max_cycles):
        residual = rhs - apply(x)
        beta = np.linalg.norm(residual)
        if callback is not None:
            callback(steps, beta / scale)
        if beta / scale < tolerance:
            return x, "converged", steps
        basis[0] = residual / beta
        h = np.zeros((restart + 1, restart), dtype=np.complex128)
        used = restart
        for j in range(restart):
            directions[j] = precondition(basis[j])
            w = apply(directions[j])
            steps += 1
            for _ in range(2):
                coefficients = basis[: j + 1].conj() @ w
                w = w - basis[: j + 1].T @ coefficients
                h[: j + 1, j] += coefficients
            h[j + 1, j] = np.linalg.norm(w)
            if abs(h[j + 1, j]) < 1e-12:
                used = j + 1
                break
            basis[j + 1] = w / h[j + 1, j]
        target = np.zeros(used + 1, dtype=np.complex128)
        target[0] = beta
        y = np.linalg.lstsq(h[: used + 1, :used], target, rcond=None)[0]
        x = x + directions[:used].T @ y
    final = float(np.linalg.norm(rhs - apply(x)) / scale)
    if callback is not None:
        callback(steps, final)
    return x, ("converged" if final < tolerance else "iteration_budget"), steps


def material_gradient(spec: Spec, c, rho, alpha_db, frequency_hz, u, lam):
    """Gradient w.r.t. ``log c`` and ``log rho`` (see :func:`material_gradient_planes`)."""
    return material_gradient_planes(spec, *material(spec, c, rho, alpha_db), frequency_hz, u, lam)


def material_gradient_planes(spec: Spec, a, b, t, frequency_hz, u, lam):
    """Gradient of a real misfit w.r.t. ``log c`` and ``log rho``.

    For ``A(m) u = s`` with ``s`` independent of the material and an adjoint
    field ``lam`` solving ``A^H lam = dL/du*``, the derivative is
    ``dL/dm = -Re(lam^H (dA/dm) u)`` -- the contraction that
    theranostic/wave.py:371-389 forms column by column (mass part
    ``k0^2 cell_mass u u`` and flux part ``-stretch edge_avg grad u grad u``) and
    that nsrno/dense_wave.py:250-255 obtains by autograd.
    Returns ``(g_logc[nz,nx], g_logrho[nz,nx])`` in float64.
    """
    nz, nx = spec.nz, spec.nx
    u = np.asarray(u, dtype=np.complex128).reshape(nz, nx)
    lam = np.asarray(lam, dtype=np.complex128).reshape(nz, nx)
    a, b, t = (np.asarray(v, dtype=np.float64) for v in (a, b, t))
    sx, sz, sxh, szh = stretches(spec, frequency_hz)
    e = t * (frequency_hz / 1e6) ** (spec.alpha_power - 1.0)
    k2 = k0_of(spec, frequency_hz) ** 2
    cell = k2 * sz[:, None] * sx[None, :] * b
    lu = lam.conj() * u
    # d mass / d log c = -2 k0^2 sxsz b (1+ie) ; d mass / d log rho = -mass
    g_c = -np.real(lu * (-2.0 * cell * (1.0 + 1j * e)))
    g_r = -np.real(lu * (-cell * (1.0 + 1j * e) ** 2))
    # Edge terms: each edge (i,j) contributes F * conj(lam_i - lam_j) (u_j - u_i)
    # = -F * conj(dlam) du to lam^H A u; dF/dlog rho_i = -stretch a_i / (2 h^2).
    # The derivative of that term is therefore +a_i w conj(dlam) du.
    up = np.pad(u, 1)
    lp = np.pad(lam, 1)
    wx = (sz[:, None] / sxh[None, :]) / (2 * spec.h ** 2)      # [nz, nx+1]
    wz = (sx[None, :] / szh[:, None]) / (2 * spec.h ** 2)      # [nz+1, nx]
    dux = up[1:-1, 1:] - up[1:-1, :-1]                         # u_{j} - u_{j-1}, [nz, nx+1]
    dlx = (lp[1:-1, 1:] - lp[1:-1, :-1]).conj()
    duz = up[1:, 1:-1] - up[:-1, 1:-1]
    dlz = (lp[1:, 1:-1] - lp[:-1, 1:-1]).conj()
    ex = wx * dlx * dux                                        # per edge, without -a_i
    ez = wz * dlz * duz
    edge_sum = ex[:, :-1] + ex[:, 1:] + ez[:-1, :] + ez[1:, :]
    g_r += -np.real(a * edge_sum)
    return g_c, g_r


def time_lu_frequency(spec: Spec, c, rho, alpha_db, frequency_hz, angles_rad):
    """Reference CPU path for one frequency: assemble, factor once, solve every angle.

    Mirrors theranostic/wave.py:252-265 (one SuperLU per frequency shared by
    all sources).  Returns ``(fields[A, n], seconds, max relative residual)``.
    """
    started = time.perf_counter()
    matrix = operator(spec, c, rho, alpha_db, frequency_hz)
    lu = splu(matrix.tocsc())
    rhs = np.stack([plane_wave_rhs(spec, frequency_hz, th) for th in angles_rad], axis=1)
    fields = lu.solve(rhs)
    seconds = time.perf_counter() - started
    res = max(relative_residual(matrix, fields[:, k], rhs[:, k]) for k in range(rhs.shape[1]))
    return fields.T, seconds, res


def operator_derivative(spec: Spec, c, rho, alpha_db, frequency_hz, dlogc, dlogrho):
    """``dA = sum_k (dA/dlog c_k) dlogc_k + (dA/dlog rho_k) dlogrho_k`` (CSR, SI).

    The directional derivative of :func:`operator` that ``born_data`` applies
    as ``delta_A`` (theranostic/wave.py:280-329, ``matrix(m) - matrix(0)`` is
    this derivative for its linear contrasts): mass ``-2 k0^2 sx sz b (1+ie)``
    per unit log c (the attenuation term is proportional to c) and ``-mass``
    per unit log rho; edge fluxes ``stretch (da_i + da_j)/(2 h^2)`` with
    ``da = -a dlogrho`` and zero ghost contrast.
    """
    a, b, t = material(spec, c, rho, alpha_db)
    dlogc = np.asarray(dlogc, dtype=np.float64)
    dlogrho = np.asarray(dlogrho, dtype=np.float64)
    sx, sz, sxh, szh = stretches(spec, frequency_hz)
    e = t * (frequency_hz / 1e6) ** (spec.alpha_power - 1.0)
    cell = k0_of(spec, frequency_hz) ** 2 * (sz[:, None] * sx[None, :]) * b
    dmass = -2.0 * cell * (1.0 + 1j * e) * dlogc - cell * (1.0 + 1j * e) ** 2 * dlogrho
    da = np.pad(-a * dlogrho, 1)                    # zero ghost contrast: no ghost derivative
    dax = 0.5 * (da[1:-1, :-1] + da[1:-1, 1:])      # [nz, nx+1]
    daz = 0.5 * (da[:-1, 1:-1] + da[1:, 1:-1])      # [nz+1, nx]
    fx = (sz[:, None] / sxh[None, :]) * dax / spec.h ** 2
    fz = (sx[None, :] / szh[:, None]) * daz / spec.h ** 2
    diagonal = dmass - fx[:, :-1] - fx[:, 1:] - fz[:-1, :] - fz[1:, :]
    nz, nx = spec.nz, spec.nx
    east_full = np.zeros((nz, nx), dtype=np.complex128)
    east_full[:, :-1] = fx[:, 1:-1]
    e1 = east_full.ravel()[:-1]
    south = fz[1:-1, :].ravel()
    return sparse.diags([diagonal.ravel(), e1, e1, south, south], [0, 1, -1, nx, -nx],
                        shape=(spec.n, spec.n), format="csr", dtype=np.complex128)


def born_fields(spec: Spec, c, rho, alpha_db, frequency_hz, u, dlogc, dlogrho):
    """Tangent fields ``du = -A^-1 dA u`` (theranostic/wave.py:280-329) by SuperLU; ``u`` is [n] or [n, k]."""
    A = operator(spec, c, rho, alpha_db, frequency_hz)
    dA = operator_derivative(spec, c, rho, alpha_db, frequency_hz, dlogc, dlogrho)
    return solve_lu(A, -(dA @ np.asarray(u, dtype=np.complex128)))
