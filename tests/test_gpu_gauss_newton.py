"""Tangent (Born) right-hand side, Jacobian-vector product, adjoint consistency
and the Gauss-Newton Hessian-vector product against the oracle."""
import numpy as np
import pytest
import torch

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu


def case(dev, seed=5):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=seed, nz=96, nx=128, n_pml=12, n_rx=24, rx_pitch=4, bins=[4.5e6, 7.2e6], n_angles=2)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=dev)
    rng = np.random.default_rng(seed)
    zz, xx = np.meshgrid(np.arange(rec.nz), np.arange(rec.nx), indexing="ij")
    win = np.exp(-((zz - 60) ** 2 + (xx - 64) ** 2) / (2 * 10.0 ** 2))
    dc = rng.standard_normal() * win * 0.02 + 0.003 * rng.standard_normal((rec.nz, rec.nx)) * rec.interior()
    dr = rng.standard_normal() * win * 0.01 + 0.002 * rng.standard_normal((rec.nz, rec.nx)) * rec.interior()
    return rec, med, dc, dr


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_tangent_rhs_matches_oracle_derivative(cuda, dtype):
    from nsrno_b200.gauss_newton import tangent_rhs
    rec, med, dc, dr = case(cuda)
    spec = spec_of(rec)
    rng = np.random.default_rng(2)
    u = rng.standard_normal((2, rec.nz, rec.nx)) + 1j * rng.standard_normal((2, rec.nz, rec.nx))
    out = tangent_rhs(med, rec.frequencies, torch.as_tensor(u, device=cuda).to(dtype), dc, dr).cpu().numpy()
    for s, f in enumerate(rec.frequencies):
        dA = H.operator_derivative(spec, rec.c, rec.rho, rec.alpha, f, dc, dr)
        want = -(dA @ u[s].ravel().astype(dtype == torch.complex64 and np.complex64 or np.complex128))
        assert rel(out[s].ravel(), want) < (1e-12 if dtype == torch.complex128 else 2e-6)


def test_jvp_matches_oracle_born_fields(cuda):
    from nsrno_b200 import solve_batched
    from nsrno_b200.gauss_newton import GaussNewton
    rec, med, dc, dr = case(cuda)
    spec = spec_of(rec)
    f, th = rec.systems()
    d_obs = torch.zeros((len(f), len(rec.rx_cols)), dtype=torch.complex128, device=cuda)
    gn = GaussNewton(med, f, th, d_obs, tolerance=1e-9)
    gn.forward()
    jv = gn.jvp(dc, dr).cpu().numpy()
    for s in range(len(f)):
        A = H.operator(spec, rec.c, rec.rho, rec.alpha, f[s])
        u = H.solve_lu(A, H.plane_wave_rhs(spec, f[s], th[s]))
        du = H.born_fields(spec, rec.c, rec.rho, rec.alpha, f[s], u, dc, dr)
        assert rel(jv[s], H.receivers(spec, du)) < 1e-5


def test_adjoint_consistency_and_hessian_symmetry(cuda):
    """<J v, r> = <v, J^H r> (real parts) and <v1, H v2> = <H v1, v2>."""
    from nsrno_b200.gauss_newton import GaussNewton
    rec, med, dc, dr = case(cuda)
    f, th = rec.systems()
    rng = np.random.default_rng(9)
    n_rx = len(rec.rx_cols)
    d_obs = torch.as_tensor(rng.standard_normal((len(f), n_rx)) + 1j * rng.standard_normal((len(f), n_rx)),
                            device=cuda) * 1e-3
    gn = GaussNewton(med, f, th, d_obs, tolerance=1e-10)
    gn.forward()
    gc, gr = gn.gradient()                       # Re(J^H r)
    jv = gn.jvp(dc, dr)
    lhs = float((jv.conj() * gn.r).real.sum())
    rhs = float((gc.cpu().numpy() * dc).sum() + (gr.cpu().numpy() * dr).sum())
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)
    _, _, dc2, dr2 = case(cuda, seed=8)
    (h1c, h1r), _ = gn.hessian_vector(dc, dr)
    (h2c, h2r), _ = gn.hessian_vector(dc2, dr2)
    a = float((h2c.cpu().numpy() * dc).sum() + (h2r.cpu().numpy() * dr).sum())
    b = float((h1c.cpu().numpy() * dc2).sum() + (h1r.cpu().numpy() * dr2).sum())
    assert abs(a - b) < 1e-5 * abs(a)


def test_gauss_newton_step_with_learned_preconditioner(cuda):
    """A full step (forward, gradient, Hessian-vector, step length) with the
    learned preconditioner equals the fixed-preconditioner step, and the
    quadratic model's predicted decrease is positive."""
    from nsrno_b200 import LearnedPreconditioner, solve_batched
    from nsrno_b200.gauss_newton import GaussNewton
    from nsrno_b200.media import perturbed
    rec, med, _, _ = case(cuda)
    f, th = rec.systems()
    from nsrno_b200 import Geometry, Medium
    true = perturbed(rec, seed=3, window=3e-3)
    obs = solve_batched(Medium(Geometry.from_record(true), true.c, true.rho, true.alpha, device=cuda), f, th,
                        tolerance=1e-10)
    steps = []
    for pre in (None, LearnedPreconditioner.load(device=cuda)):
        gn = GaussNewton(med, f, th, obs.iq, preconditioner=pre, tolerance=1e-9)
        steps.append(gn.step())
    assert steps[0]["predicted_decrease"] > 0
    assert abs(steps[1]["alpha"] - steps[0]["alpha"]) < 1e-5 * abs(steps[0]["alpha"])
    assert rel(steps[1]["update"][0].cpu().numpy(), steps[0]["update"][0].cpu().numpy()) < 1e-5
