"""GPU restarted GMRES against the SuperLU oracle and against the oracle's
restatement of the reference GMRES cycle (nsrno/wave_solver.py:9-36)."""
import math

import numpy as np
import pytest
import torch

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu


def blob_case(dev):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import blob_record
    rec = blob_record()
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=dev)
    return rec, med


def fft_preconditioner(rec, f, shift=0.15):
    kh2 = (2 * math.pi * f / rec.c0 * rec.h) ** 2
    qz = np.sin(np.pi * np.arange(rec.nz) / rec.nz) ** 2
    qx = np.sin(np.pi * np.arange(rec.nx) / rec.nx) ** 2
    mul = 1.0 / (-4.0 * (qz[:, None] + qx[None, :]) + kh2 * (1 + 1j * shift))
    return lambda v: np.fft.ifft2(np.fft.fft2(v.reshape(rec.nz, rec.nx)) * mul).ravel()


def test_gmres_converges_to_lu(cuda):
    from nsrno_b200 import gmres_batched
    rec, med = blob_case(cuda)
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    f, th = rec.systems()
    res = gmres_batched(med, f, th, tolerance=1e-7, restart=32, max_iterations=3200, n_slots=4, return_fields=True)
    assert res.reasons() == ["converged"] * len(f)
    assert float(res.residual.max()) < 1e-7
    for s in range(len(f)):
        ref = H.solve_lu(H.operator_planes(spec, a, b, t, f[s]), H.plane_wave_rhs(spec, f[s], th[s]))
        assert rel(res.fields[s].cpu().numpy().ravel(), ref) < 1e-5
        assert rel(res.iq[s].cpu().numpy(), H.receivers(spec, ref)) < 1e-5


def test_one_cycle_matches_reference_gmres(cuda):
    """One GMRES(12) cycle on the GPU equals one cycle of the restated reference loop."""
    from nsrno_b200 import gmres_batched
    rec, med = blob_case(cuda)
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    f, th = 1.5e6, rec.angles[0]
    A = H.operator_planes(spec, a, b, t, f) * rec.h ** 2
    rhs = H.plane_wave_rhs(spec, f, th) * rec.h ** 2
    x_ref, reason, steps = H.gmres(lambda v: A @ v, rhs, restart=12, max_cycles=1, tolerance=1e-30,
                                   precondition=fft_preconditioner(rec, f))
    res = gmres_batched(med, [f], [th], tolerance=1e-30, restart=12, max_iterations=12, return_fields=True,
                        fields_dtype=torch.complex128)
    assert int(res.iterations[0]) == 12 and res.reasons() == ["iteration_budget"]
    assert rel(res.fields[0].cpu().numpy().ravel(), x_ref) < 1e-5
    assert abs(float(res.residual[0]) - H.relative_residual(A, x_ref, rhs)) < 1e-5 * float(res.residual[0])


def test_adjoint_gmres_matches_lu(cuda):
    from nsrno_b200 import gmres_batched
    rec, med = blob_case(cuda)
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    rng = np.random.default_rng(9)
    g = np.zeros((1, rec.nz, rec.nx), np.complex64)
    g[0, rec.face, rec.rx_cols] = rng.standard_normal(len(rec.rx_cols)) + 1j * rng.standard_normal(len(rec.rx_cols))
    f = 1.0e6
    res = gmres_batched(med, [f], rhs=torch.as_tensor(g, device=cuda), adjoint=True, tolerance=1e-8,
                        max_iterations=3200, return_fields=True)
    ref = H.solve_lu(H.operator_planes(spec, a, b, t, f).conj().T.tocsc(), g[0].ravel().astype(np.complex128))
    assert res.reasons() == ["converged"]
    assert rel(res.fields[0].cpu().numpy().ravel(), ref) < 1e-5


def test_gmres_batches_and_budget(cuda):
    """More systems than slots run in batches; an exhausted budget is reported."""
    from nsrno_b200 import gmres_batched, solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    r = gmres_batched(med, f, th, tolerance=1e-6, restart=24, max_iterations=2400, n_slots=2)
    assert r.reasons() == ["converged"] * len(f)
    b = solve_batched(med, f, th, tolerance=1e-6)
    assert rel(r.iq.cpu().numpy(), b.iq.cpu().numpy()) < 1e-4
    r = gmres_batched(med, f[:2], th[:2], tolerance=1e-12, restart=8, max_iterations=16)
    assert r.reasons() == ["iteration_budget"] * 2
    assert (r.iterations.cpu() == 16).all()
