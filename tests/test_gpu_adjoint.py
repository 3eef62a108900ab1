"""Adjoint solve + gradient kernel: against the reference Born Jacobian (golden)
and against central differences of the oracle (the config-3 check)."""
import math

import numpy as np
import pytest
import torch
from scipy import sparse

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu


def test_gradient_matches_reference_born_jacobian(cuda, golden):
    """Re(J^H r) of theranostic/wave.py:331-389 (tests/test_theranostic.py:108-114) from one
    forward and one adjoint solve per transmitter plus the fused gradient kernel."""
    from nsrno_b200 import Geometry, Medium, grad_accum, solve_batched
    axis = golden["fixture_axis_mm"]
    h = float(axis[1] - axis[0]) * 1e-3
    n = axis.size
    geo = Geometry(nz=n, nx=n, h=h, n_pml=int(round(6.0 / (h * 1e3))), face=0, rx_cols=np.arange(1),
                   aperture_half_width=0.0, c0=float(golden["fixture_c0"]))
    ones = np.ones((n, n), np.float32)
    med = Medium(geo, ones * geo.c0, ones * geo.rho0, ones * 0.0, device=cuda)
    W = sparse.csc_matrix((golden["weights_val"], (golden["weights_row"], golden["weights_col"])), shape=(n * n, 4))
    f = float(golden["fixture_freq_mhz"]) * 1e6
    Wd = W.toarray()
    rhs = (-(Wd.T) / h ** 2).reshape(4, n, n).astype(np.complex64)
    fwd = solve_batched(med, [f] * 4, rhs=torch.as_tensor(rhs, device=cuda), tolerance=1e-9, return_fields=True,
                        fields_dtype=torch.complex128)
    r = golden["residual"].reshape(4, 4)                       # [tx, rx]
    adj_rhs = (Wd @ r.T).T.reshape(4, n, n).astype(np.complex64)   # P^T r per transmitter
    adj = solve_batched(med, [f] * 4, rhs=torch.as_tensor(adj_rhs, device=cuda), tolerance=1e-9, adjoint=True,
                        return_fields=True, fields_dtype=torch.complex128)
    assert fwd.reasons() == ["converged"] * 4 and adj.reasons() == ["converged"] * 4
    g_logc, g_logrho = grad_accum(med, [f] * 4, fwd.fields, adj.fields)
    g_logc = g_logc.cpu().numpy().ravel()
    g_logrho = g_logrho.cpu().numpy().ravel()
    # at zero contrast: b = 1 + m_kappa, a = 1 + m_eta, db/dlogc = -2, db/dlogrho = -1, da/dlogrho = -1
    d_mk = -g_logc / 2.0
    d_me = -g_logrho - d_mk
    basis = golden["basis"]
    ours = np.concatenate((basis.T @ d_mk, basis.T @ d_me))
    assert rel(ours, golden["gradient"]) < 1e-6


def config3_case(dev):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import blob_record, perturbed
    rec = blob_record()
    true = perturbed(rec, seed=3)
    return rec, true


def oracle_misfit(spec, c, rho, alpha, systems, d_obs):
    total = 0.0
    for (f, th), d in zip(systems, d_obs):
        A = H.operator(spec, c, rho, alpha, f)
        u = H.solve_lu(A, H.plane_wave_rhs(spec, f, th))
        r = H.receivers(spec, u) - d
        total += 0.5 * float(np.vdot(r, r).real)
    return total


def test_config3_gradient_against_central_differences(cuda):
    """L2 IQ misfit of the 256x256 record against data of a perturbed medium:
    GPU implicit gradient vs oracle central differences (step 1e-3) at 16 random
    pixels and along 4 random directions (Richardson-extrapolated with step 5e-4),
    tolerance 1e-4 relative."""
    from nsrno_b200 import AcquisitionData, Geometry, implicit_channels
    rec, true = config3_case(cuda)
    spec = spec_of(rec)
    f, th = rec.systems()
    systems = list(zip(f, th))
    # observed data from the perturbed medium, by the oracle (complex128)
    d_obs = []
    for fr, an in systems:
        A = H.operator(spec, true.c, true.rho, true.alpha, fr)
        d_obs.append(H.receivers(spec, H.solve_lu(A, H.plane_wave_rhs(spec, fr, an))))
    geo = Geometry.from_record(rec)
    data = AcquisitionData(geo, np.rad2deg(rec.angles), response=False)
    medium = torch.as_tensor(np.stack((rec.c, rec.rho)).astype(np.float64), device=cuda).requires_grad_(True)
    alpha = torch.as_tensor(rec.alpha.astype(np.float64), device=cuda)
    loss = 0.0
    for k, fr in enumerate(rec.frequencies):
        out = implicit_channels(medium, alpha, data, float(fr), [0, 1, 2], tolerance=1e-10)
        obs = torch.as_tensor(np.stack(d_obs[3 * k:3 * k + 3]), device=cuda)
        loss = loss + 0.5 * (out - obs).abs().square().sum()
    loss.backward()
    grad = medium.grad.cpu().numpy()            # d/dc, d/drho
    g_logc = grad[0] * rec.c.astype(np.float64)
    g_logrho = grad[1] * rec.rho.astype(np.float64)
    rng = np.random.default_rng(3)
    interior = np.argwhere(rec.interior())
    c0 = rec.c.astype(np.float64)
    r0 = rec.rho.astype(np.float64)
    eps = 1e-3

    def central(dc, dr, h):
        lp = oracle_misfit(spec, c0 * np.exp(h * dc), r0 * np.exp(h * dr), rec.alpha, systems, d_obs)
        lm = oracle_misfit(spec, c0 * np.exp(-h * dc), r0 * np.exp(-h * dr), rec.alpha, systems, d_obs)
        return (lp - lm) / (2 * h)

    def fd(dc, dr):
        # Central differences at step 1e-3 carry an O(h^2) truncation error of
        # about 1e-4 on this record; Richardson extrapolation with h/2 removes it.
        return (4.0 * central(dc, dr, eps / 2) - central(dc, dr, eps)) / 3.0

    # random directions (smooth windows) over both parameters
    xx, zz = np.meshgrid(np.arange(rec.nx), np.arange(rec.nz))
    for _ in range(4):
        cz, cx = interior[rng.integers(len(interior))]
        win = np.exp(-((xx - cx) ** 2 + (zz - cz) ** 2) / (2 * 12.0 ** 2))
        dc, dr = rng.standard_normal() * win, rng.standard_normal() * win
        analytic = float((g_logc * dc).sum() + (g_logrho * dr).sum())
        assert abs(analytic - fd(dc, dr)) <= 1e-4 * abs(analytic)
    # single pixels
    worst = 0.0
    for _ in range(16):
        cz, cx = interior[rng.integers(len(interior))]
        which = rng.integers(2)
        d = np.zeros_like(c0)
        d[cz, cx] = 1.0
        num = fd(d, 0 * d) if which == 0 else fd(0 * d, d)
        ana = (g_logc if which == 0 else g_logrho)[cz, cx]
        worst = max(worst, abs(ana - num) / max(abs(num), 1e-30))
    assert worst < 1e-4
