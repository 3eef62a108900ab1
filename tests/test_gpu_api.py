"""Reference-facing contracts on the GPU: solve_frequency, solve_system and the
DenseSurrogate drop-in (nsrno/wave_solver.py:38-67, nsrno/dense_wave.py:167-259,
nsrno/dense_surrogate.py:9-36)."""
import numpy as np
import pytest
import torch

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu


def blob(dev):
    from nsrno_b200 import Geometry
    from nsrno_b200.media import blob_record
    rec = blob_record()
    return rec, Geometry.from_record(rec)


def oracle_iq(rec, f, th):
    spec = spec_of(rec)
    u = H.solve_lu(H.operator(spec, rec.c, rec.rho, rec.alpha, f), H.plane_wave_rhs(spec, f, th))
    return H.receivers(spec, u), u


def test_solve_frequency_contract(cuda):
    from nsrno_b200 import PlaneWaveModel, solve_frequency
    rec, geo = blob(cuda)
    model = PlaneWaveModel(geo, np.rad2deg(rec.angles), alpha=rec.alpha)
    medium = torch.as_tensor(np.stack((rec.c, rec.rho))[None], device=cuda)
    pred, status = solve_frequency(model, medium, 1.5e6, 1, tolerance=1e-6, max_iterations=2560, restart=32)
    assert set(status) >= {"reason", "initial_neural_iterations", "solver_iterations", "relative_residual",
                           "seconds", "trace"}
    assert status["reason"] == "converged" and status["relative_residual"] < 1e-6
    assert pred.dtype == torch.complex64 and pred.shape == (192,)
    ref, _ = oracle_iq(rec, 1.5e6, rec.angles[1])
    assert rel(pred.cpu().numpy(), ref) < 1e-4


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
def test_solve_system_contract(cuda, method):
    from nsrno_b200 import HelmholtzSystem, Medium, plane_wave_rhs, solve_system
    rec, geo = blob(cuda)
    med = Medium(geo, rec.c, rec.rho, rec.alpha, device=cuda)
    f = 1.0e6
    rhs = plane_wave_rhs(med, [f] * 3, rec.angles)
    x, info = solve_system(HelmholtzSystem(med, f), rhs, tolerance=1e-7, method=method)
    assert set(info) >= {"reason", "steps", "residual", "max_angle_residual", "seconds", "dtype", "method"}
    assert info["reason"] == "converged" and info["max_angle_residual"] < 1e-7
    for k in range(3):
        _, u = oracle_iq(rec, f, rec.angles[k])
        assert rel(x[k].cpu().numpy().ravel(), u) < 1e-5


def test_surrogate_forward_backward_and_truncated(cuda):
    from nsrno_b200 import HelmholtzSurrogate, bin_frequency
    rec, geo = blob(cuda)
    # a 256x256 record at 0.1 mm with bins in the 1 MHz range of this grid
    sur = HelmholtzSurrogate(geo, np.rad2deg(rec.angles), bins=[60, 61], response=False)
    medium = torch.as_tensor(np.stack((rec.c, rec.rho)).astype(np.float64), device=cuda).requires_grad_(True)
    alpha = torch.as_tensor(rec.alpha.astype(np.float64), device=cuda)
    out = sur(medium, alpha, 60, tolerance=1e-8)
    assert out.shape == (3, 192) and out.dtype == torch.complex128
    ref = np.stack([oracle_iq(rec, bin_frequency(60), th)[0] for th in rec.angles])
    assert rel(out.detach().cpu().numpy(), ref) < 1e-5
    out.abs().square().sum().backward()
    assert torch.isfinite(medium.grad).all() and float(medium.grad.abs().max()) > 0
    ch, res = sur.truncated(medium.detach(), alpha, 60, iterations=4)
    assert ch.shape == (3, 192) and 0 < res < 1
    with pytest.raises(RuntimeError, match="Forward failed to converge"):
        from nsrno_b200 import AcquisitionData, implicit_channels
        implicit_channels(medium, alpha, AcquisitionData(geo, np.rad2deg(rec.angles), response=False),
                          bin_frequency(60), [0], tolerance=1e-12, max_iterations=2)


def small_breast(dev):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=31, nz=128, nx=192, n_pml=16, n_rx=40, rx_pitch=4, n_angles=3)
    return rec, Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=dev)


@pytest.mark.parametrize("method", ["bicgstab", "gmres_learned"])
def test_solve_system_with_learned_preconditioner(cuda, method):
    """The learned preconditioner with the reference's 8-step warm start
    (nsrno/dense_wave.py:197-208): same solution as SuperLU, warm steps counted."""
    from nsrno_b200 import HelmholtzSystem, LearnedPreconditioner, plane_wave_rhs, solve_system
    rec, med = small_breast(cuda)
    f = float(rec.frequencies[200])
    rhs = plane_wave_rhs(med, [f] * 3, rec.angles)
    net = LearnedPreconditioner.load(device=cuda)
    x, info = solve_system(HelmholtzSystem(med, f), rhs, preconditioner=net, tolerance=1e-7, method=method,
                           warm_steps=8)
    assert info["reason"] == "converged" and info["max_angle_residual"] < 1e-7
    assert info["steps"] >= 3 * 8
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    A = H.operator_planes(spec, a, b, t, f)
    for k in range(3):
        u = H.solve_lu(A, H.plane_wave_rhs(spec, f, rec.angles[k]))
        assert rel(x[k].cpu().numpy().ravel(), u) < 1e-5


def test_learned_and_fixed_gradients_agree(cuda):
    """The implicit gradient does not depend on the preconditioner (forward and
    adjoint both converged): learned vs fixed on a breast-like record."""
    from nsrno_b200 import AcquisitionData, Geometry, LearnedPreconditioner, implicit_channels
    rec, med = small_breast(cuda)
    geo = Geometry.from_record(rec)
    data = AcquisitionData(geo, np.rad2deg(rec.angles), response=False)
    f = float(rec.frequencies[120])
    alpha = torch.as_tensor(rec.alpha.astype(np.float64), device=cuda)
    grads, outs = [], []
    for pre in (None, LearnedPreconditioner.load(device=cuda)):
        medium = torch.as_tensor(np.stack((rec.c, rec.rho)).astype(np.float64), device=cuda).requires_grad_(True)
        out = implicit_channels(medium, alpha, data, f, [0, 1, 2], tolerance=1e-9, preconditioner=pre)
        (out.abs().square().sum()).backward()
        grads.append(medium.grad.cpu().numpy())
        outs.append(out.detach().cpu().numpy())
    assert rel(outs[1], outs[0]) < 1e-6
    assert rel(grads[1], grads[0]) < 1e-5


def test_truncated_is_one_learned_gmres_cycle(cuda):
    """``truncated`` is one GMRES cycle of K steps with the learned
    preconditioner (nsrno/dense_surrogate.py:30-36 through batched_gmres_cycle,
    nsrno/dense_wave.py:84-116): channels and the actual residual equal the
    oracle's restated cycle (complex128, SciPy operator, oracle network)."""
    import math
    from oracle import learned_ref as L
    from nsrno_b200 import HelmholtzSurrogate, bin_frequency
    from nsrno_b200.learned import LearnedPreconditioner
    rec, med = small_breast(cuda)
    geo = med.geometry
    net = LearnedPreconditioner.load(device=cuda)
    sur = HelmholtzSurrogate(geo, np.rad2deg(rec.angles), bins=[300], response=False, preconditioner=net)
    medium = torch.as_tensor(np.stack((rec.c, rec.rho)).astype(np.float64), device=cuda)
    alpha = torch.as_tensor(rec.alpha.astype(np.float64), device=cuda)
    f = bin_frequency(300)
    K = 8
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    A = H.operator_planes(spec, a, b, t, f) * rec.h ** 2
    lp = L.Learned(net.params.double().cpu(), med.c.double().cpu(), med.rho.double().cpu(), med.alpha.double().cpu(),
                   f, rec.h, rec.c0)
    pre = lambda v: lp.apply(torch.as_tensor(v.reshape(rec.nz, rec.nx))).numpy().ravel()
    ch, res = sur.truncated(medium, alpha, 300, angles=[0, 2], iterations=K)
    rr, bb = 0.0, 0.0
    for k, a_idx in enumerate([0, 2]):
        rhs = H.plane_wave_rhs(spec, f, rec.angles[a_idx]) * rec.h ** 2
        x_ref, _, steps = H.gmres(lambda v: A @ v, rhs, restart=K, max_cycles=1, tolerance=1e-30, precondition=pre)
        assert rel(ch[k].cpu().numpy(), H.receivers(spec, x_ref)) < 1e-4
        rr += np.linalg.norm(A @ x_ref - rhs) ** 2
        bb += np.linalg.norm(rhs) ** 2
    assert abs(res - math.sqrt(rr / bb)) < 1e-4 * res
    # more steps, smaller residual
    _, res16 = sur.truncated(medium, alpha, 300, angles=[0, 2], iterations=16)
    assert res16 < res
