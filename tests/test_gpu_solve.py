"""GPU parity of the batched BiCGSTAB solve against the SuperLU oracle and the
reference's own golden vectors."""
import math

import numpy as np
import pytest
import torch
from scipy import sparse
from scipy.special import hankel1

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu


def blob_case(dev):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import blob_record
    rec = blob_record()
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=dev)
    return rec, med


def test_blob_record_matches_lu(cuda):
    """256x256 record, 3 angles x 2 frequencies: fields and receiver IQ vs SuperLU."""
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    f, th = rec.systems()
    res = solve_batched(med, f, th, tolerance=1e-7, max_iterations=2000, return_fields=True, n_slots=4)
    assert res.reasons() == ["converged"] * len(f)
    assert float(res.residual.max()) < 1e-7
    fields = res.fields.cpu().numpy()
    iq = res.iq.cpu().numpy()
    for s in range(len(f)):
        A = H.operator_planes(spec, a, b, t, f[s])
        rhs = H.plane_wave_rhs(spec, f[s], th[s])
        ref = H.solve_lu(A, rhs)
        assert rel(fields[s].ravel(), ref) < 1e-5
        assert rel(iq[s], H.receivers(spec, ref)) < 1e-5


def test_slot_refill_is_bitwise_identical(cuda):
    """Results do not depend on how many slots are resident (queue refill)."""
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    r1 = solve_batched(med, f, th, tolerance=1e-6, n_slots=1)
    r6 = solve_batched(med, f, th, tolerance=1e-6, n_slots=6)
    assert torch.equal(r1.iq, r6.iq)
    assert torch.equal(r1.iterations, r6.iterations)


def fixture_case(golden, dev):
    from nsrno_b200 import Geometry, Medium
    axis = golden["fixture_axis_mm"]
    h = float(axis[1] - axis[0]) * 1e-3
    n = axis.size
    n_pml = int(round(float(golden["fixture_pml_mm"]) * 1e-3 / h))
    geo = Geometry(nz=n, nx=n, h=h, n_pml=n_pml, face=n // 2, rx_cols=np.arange(4), aperture_half_width=0.0,
                   c0=float(golden["fixture_c0"]))
    ones = np.ones((n, n), np.float32)
    med = Medium(geo, ones * geo.c0, ones * geo.rho0, ones * 0.0, device=dev)
    W = sparse.csc_matrix((golden["weights_val"], (golden["weights_row"], golden["weights_col"])),
                          shape=(n * n, 4))
    return geo, med, W


def test_reference_fixture_fields_and_response(cuda, golden):
    """The reference unit-test fixture (81x81, four finite elements) against its own solve."""
    from nsrno_b200 import solve_batched
    geo, med, W = fixture_case(golden, cuda)
    f = float(golden["fixture_freq_mhz"]) * 1e6
    rhs = (-(W.toarray().T) / geo.h ** 2).reshape(4, geo.nz, geo.nx).astype(np.complex64)
    res = solve_batched(med, [f] * 4, rhs=torch.as_tensor(rhs, device=cuda), tolerance=1e-9,
                        max_iterations=3000, return_fields=True)
    assert res.reasons() == ["converged"] * 4
    u = res.fields.cpu().numpy().reshape(4, -1).T.astype(np.complex128)
    assert rel(u, golden["fields"]) < 1e-5
    response = (W.T @ u).T
    assert rel(response, golden["response"]) < 1e-5
    # reciprocity of the response matrix (complex symmetric, not Hermitian)
    assert rel(response, response.T) < 1e-5


def test_green_function_known_answer(cuda):
    """div grad p + k^2 p = -delta against 0.25 i H0(k r) (tests/test_theranostic.py:141-158)."""
    from nsrno_b200 import Geometry, Medium, solve_batched
    axis = np.linspace(-16.0, 16.0, 81)
    h = (axis[1] - axis[0]) * 1e-3
    n = axis.size
    geo = Geometry(nz=n, nx=n, h=h, n_pml=int(round(6.0 / (h * 1e3))), face=0, rx_cols=np.arange(1),
                   aperture_half_width=0.0, c0=1540.0)
    ones = np.ones((n, n), np.float32)
    med = Medium(geo, ones * 1540.0, ones * 1000.0, ones * 0.0, device=cuda)
    positions = np.array([[-3.2, 0.0], [3.2, 0.0], [0.0, 4.8]])
    idx = [int(round((p[1] + 16.0) / (h * 1e3))) * n + int(round((p[0] + 16.0) / (h * 1e3))) for p in positions]
    rhs = np.zeros((3, n * n), np.complex64)
    for s, k in enumerate(idx):
        rhs[s, k] = -1.0 / h ** 2
    rx = torch.as_tensor(np.array(idx, np.int32), device=cuda)
    f = 0.15e6
    res = solve_batched(med, [f] * 3, rhs=torch.as_tensor(rhs.reshape(3, n, n), device=cuda), tolerance=1e-9,
                        max_iterations=3000, rx_index=rx)
    measured = res.iq.cpu().numpy()
    off = ~np.eye(3, dtype=bool)
    d = np.linalg.norm(positions[:, None] - positions[None, :], axis=2) * 1e-3
    exact = 0.25j * hankel1(0, 2 * np.pi * f / 1540.0 * d[off])
    assert rel(measured[off], exact) < 0.02


def test_adjoint_solve_matches_lu(cuda):
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    rng = np.random.default_rng(9)
    g = np.zeros((1, rec.nz, rec.nx), np.complex64)
    g[0, rec.face, rec.rx_cols] = (rng.standard_normal(len(rec.rx_cols)) + 1j * rng.standard_normal(len(rec.rx_cols)))
    f = 1.5e6
    res = solve_batched(med, [f], rhs=torch.as_tensor(g, device=cuda), adjoint=True, tolerance=1e-8,
                        return_fields=True)
    A = H.operator_planes(spec, a, b, t, f)
    ref = H.solve_lu(A.conj().T.tocsc(), g[0].ravel().astype(np.complex128))
    assert res.reasons() == ["converged"]
    assert rel(res.fields[0].cpu().numpy().ravel(), ref) < 1e-5


def test_status_paths(cuda):
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    # iteration budget
    r = solve_batched(med, f[:2], th[:2], tolerance=1e-12, max_iterations=3)
    assert r.reasons() == ["iteration_budget"] * 2
    assert (r.iterations.cpu() == 3).all()
    assert (r.residual.cpu() > 1e-12).all()
    # zero right-hand side converges to the zero field
    z = torch.zeros((1, rec.nz, rec.nx), dtype=torch.complex64, device=cuda)
    r = solve_batched(med, [1e6], rhs=z, return_fields=True)
    assert r.reasons() == ["converged"]
    assert float(r.fields.abs().max()) == 0.0
    # non-finite right-hand side is reported, not trapped
    bad = torch.zeros((1, rec.nz, rec.nx), dtype=torch.complex64, device=cuda)
    bad[0, 5, 5] = float("nan")
    r = solve_batched(med, [1e6], rhs=bad)
    assert r.reasons() == ["nonfinite"]


def test_warm_start_from_solution_needs_no_iterations(cuda):
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    r = solve_batched(med, f[:3], th[:3], tolerance=1e-7, return_fields=True)
    w = solve_batched(med, f[:3], th[:3], tolerance=1e-5, x0=r.fields.contiguous())
    assert w.reasons() == ["converged"] * 3
    assert (w.iterations.cpu() == 0).all()


def test_warm_start_gate_discards_bad_initial_fields(cuda):
    """An initial field whose relative residual exceeds the gate (1.0) is dropped:
    the system then runs exactly like a zero start (config 4's fallback rule)."""
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    cold = solve_batched(med, f[:3], th[:3], tolerance=1e-6)
    rng = np.random.default_rng(4)
    noise = torch.as_tensor((rng.standard_normal((3, rec.nz, rec.nx)) * 1e3).astype(np.complex64), device=cuda)
    bad = solve_batched(med, f[:3], th[:3], tolerance=1e-6, x0=noise, blocking=True)
    assert bad.extra["stats"]["warm_rejected"] == 3 and bad.extra["stats"]["warm_accepted"] == 0
    assert torch.equal(bad.iterations, cold.iterations)
    assert torch.equal(bad.iq, cold.iq)
    ok = solve_batched(med, f[:3], th[:3], tolerance=1e-6, x0=noise, warm_gate=0.0, blocking=True)
    assert ok.extra["stats"]["warm_accepted"] == 3 and ok.reasons() == ["converged"] * 3


def test_growing_residual_restarts(cuda):
    """The one system of 24,000 training-media solves whose FP32 recurrence ran
    away (relative residual 1.3e5 at iteration 320) converges once a growing
    true residual restarts the recurrence."""
    from nsrno_b200 import Geometry, Medium, solve_batched
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=106, nz=256, nx=384, n_rx=88, rx_pitch=4)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f = [8796334.860474803] * 2
    th = [0.17115545431964527, -0.2]
    res = solve_batched(med, f, th, tolerance=1e-6, max_iterations=6000, n_slots=2)
    assert res.reasons() == ["converged"] * 2
    assert float(res.residual.max()) < 1e-6


def test_empty_batch(cuda):
    from nsrno_b200 import gmres_batched, solve_batched
    rec, med = blob_case(cuda)
    r = solve_batched(med, [], [])
    assert r.iq.shape[0] == 0 and r.reasons() == []
    g = gmres_batched(med, [], [])
    assert g.reasons() == []


def test_odd_width_grid_matches_lu(cuda):
    """243 x 729 (odd widths: the one-column stencil kernel), fixed and learned
    preconditioners, against SuperLU."""
    from nsrno_b200 import Geometry, LearnedPreconditioner, Medium, solve_batched
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=9, nz=243, nx=729, n_pml=20, n_rx=64, rx_pitch=4, bins=[5.2e6], n_angles=2)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    A = H.operator_planes(spec, a, b, t, f[0])
    st = LearnedPreconditioner.load(device=cuda).setup(med, rec.frequencies)
    for learned in (None, st):
        res = solve_batched(med, f, th, tolerance=1e-8, max_iterations=4000, return_fields=True, learned=learned)
        assert res.reasons() == ["converged"] * 2
        for s in range(2):
            ref = H.solve_lu(A, H.plane_wave_rhs(spec, f[s], th[s]))
            assert rel(res.fields[s].cpu().numpy().ravel(), ref) < 1e-5


def test_largest_grid_converges(cuda):
    """2048 x 2048, the largest transform size (8-column tiles in the column
    pass): converged systems whose FP64 true residual, recomputed by the
    independent nsr_true_residual kernel, meets the tolerance."""
    from nsrno_b200 import Geometry, Medium, solve_batched, true_residual
    from nsrno_b200.media import blob_record
    rec = blob_record(nz=2048, nx=2048, h=5e-5, n_pml=32, n_blobs=4, frequencies=(1.5e6,), n_rx=192, rx_pitch=4)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    res = solve_batched(med, f[:2], th[:2], tolerance=1e-6, max_iterations=4000, return_fields=True,
                        fields_dtype=torch.complex128)
    assert res.reasons() == ["converged"] * 2
    tr = true_residual(med, res.fields, f[:2], th[:2]).cpu().numpy()
    assert (tr < 1e-6).all()
    assert np.allclose(tr, res.residual.cpu().numpy(), rtol=1e-6)


def test_even_width_not_multiple_of_four_matches_lu(cuda):
    """96 x 54 (even, not a multiple of 4: the two-column register stencil
    instead of the ring-staged one) against SuperLU."""
    from nsrno_b200 import Geometry, Medium, solve_batched
    from nsrno_b200.media import blob_record
    rec = blob_record(nz=96, nx=54, h=1e-4, n_pml=8, n_blobs=2, frequencies=(1.2e6,), n_rx=16, rx_pitch=2)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    res = solve_batched(med, f, th, tolerance=1e-9, max_iterations=3000, return_fields=True)
    assert res.reasons() == ["converged"] * len(f)
    A = H.operator_planes(spec, a, b, t, f[0])
    for s in range(len(f)):
        ref = H.solve_lu(A, H.plane_wave_rhs(spec, f[s], th[s]))
        assert rel(res.fields[s].cpu().numpy().ravel(), ref) < 1e-5


def test_time_limit_reports_timeout(cuda):
    """A per-system time limit that runs out ends the system with reason
    'timeout' and the FP64 true residual of the iterate it reached; systems
    that converge first are unaffected."""
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    r = solve_batched(med, f[:2], th[:2], tolerance=1e-12, max_iterations=4000, time_limit=1e-6)
    assert r.reasons() == ["timeout"] * 2
    res = r.residual.cpu().numpy()
    assert np.all(np.isfinite(res)) and np.all(res < 1.0)
    assert (r.iterations.cpu() < 40).all()
    ok = solve_batched(med, f[:2], th[:2], tolerance=1e-6, time_limit=60.0)
    assert ok.reasons() == ["converged"] * 2


@pytest.mark.parametrize("tiles", [
    dict(cols_width=8, row_tile=2, slot_groups=1),
    dict(slot_groups=3),
    dict(slot_groups=4, row_tile=8),
    dict(cols_staged=1),
    dict(rows_staged=1),
    dict(cols_staged=1, rows_staged=1, row_tile=8),
    dict(stencil_width=512, stencil_depth=4, stencil_rows=8),
    dict(stencil_width=512, stencil_depth=4, stencil_cols=2, stencil_rows=32, stencil_ctas=1),
    dict(stencil_width=256, stencil_depth=6, stencil_cols=2, stencil_rows=4, slot_groups=1),
    dict(stencil_width=256, stencil_depth=4, stencil_cols=1, stencil_rows=64),
    dict(stencil_depth=4, stencil_rows=32),
])
def test_launch_shapes_agree(cuda, tiles):
    """Every launch shape the autotuner may pick solves the same systems.  Shapes
    of the transforms and of the slot groups leave each slot's arithmetic as it
    is (bitwise equal); stencil shapes regroup the FP64 partial sums of the
    inner products, so those agree to the solve tolerance."""
    from nsrno_b200 import solve_batched
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    base = solve_batched(med, f, th, tolerance=1e-7, n_slots=6, max_iterations=3000)
    got = solve_batched(med, f, th, tolerance=1e-7, n_slots=6, max_iterations=3000, tiles=tiles)
    assert got.reasons() == ["converged"] * len(f)
    if not any(k.startswith("stencil") for k in tiles):
        assert torch.equal(got.iq, base.iq) and torch.equal(got.iterations, base.iterations)
    else:
        assert rel(got.iq.cpu().numpy(), base.iq.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("tiles", [None, dict(stencil_width=512, stencil_depth=4), dict(stencil_rows=16),
                                   dict(stencil_rows=32, stencil_depth=5), dict(slot_groups=4)])
def test_two_slot_groups_are_deterministic(cuda, tiles):
    """Twenty-two systems of the 1024 x 768 breast record, two slot groups on
    concurrent graph branches, exactly ten iterations: two runs of one launch
    shape give bitwise equal FP64 residuals.  A stencil ring that handed a row
    buffer back before its shared-memory loads had landed made these shapes
    differ from run to run."""
    from nsrno_b200 import Geometry, Medium, solve_batched
    from nsrno_b200.media import breast_record
    rec = breast_record()
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, a = rec.systems()
    pick = np.linspace(0, len(f) - 1, 22).round().astype(int)
    runs = [solve_batched(med, f[pick], a[pick], tolerance=1e-30, max_iterations=10, n_slots=22, tiles=tiles,
                          blocking=True).residual.cpu() for _ in range(3)]
    assert torch.equal(runs[0], runs[1]) and torch.equal(runs[0], runs[2])


def test_grid_with_prime_factors_matches_lu(cuda):
    """110 x 140 = (2 5 11) x (4 5 7): transforms with direct-DFT prime stages
    in both directions, fixed and learned preconditioners, against SuperLU."""
    from nsrno_b200 import Geometry, LearnedPreconditioner, Medium, solve_batched
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=12, nz=110, nx=140, n_pml=12, n_rx=32, rx_pitch=4, bins=[5.6e6], n_angles=2)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    A = H.operator_planes(spec, a, b, t, f[0])
    st = LearnedPreconditioner.load(device=cuda).setup(med, rec.frequencies)
    for learned in (None, st):
        res = solve_batched(med, f, th, tolerance=1e-8, max_iterations=4000, return_fields=True, learned=learned)
        assert res.reasons() == ["converged"] * 2
        for s in range(2):
            ref = H.solve_lu(A, H.plane_wave_rhs(spec, f[s], th[s]))
            assert rel(res.fields[s].cpu().numpy().ravel(), ref) < 1e-5


def test_device_loop_equals_host_loop(cuda):
    """The non-blocking solve (one graph launch whose conditional WHILE node
    repeats the iterations until the queue is empty) gives bitwise the results
    of the host-polled loop, and its progress record accounts for every system."""
    from nsrno_b200 import solve_batched
    from nsrno_b200.solver import solve_progress
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    for k in (16, 7, 1):   # loop rounds of several lengths: a system may finish on any iteration of a round
        host = solve_batched(med, f, th, tolerance=1e-7, n_slots=4, blocking=True, return_fields=True,
                             graph_iterations=k)
        dev = solve_batched(med, f, th, tolerance=1e-7, n_slots=4, blocking=False, return_fields=True,
                            graph_iterations=k)
        torch.cuda.synchronize()
        assert not dev.extra["blocking"] and host.extra["blocking"]
        assert torch.equal(dev.iq, host.iq) and torch.equal(dev.iterations, host.iterations)
        assert torch.equal(dev.status, host.status) and torch.equal(dev.residual, host.residual)
        # every field was emitted before the device loop ended
        assert torch.equal(dev.fields, host.fields)
    done, rounds, error, launches = solve_progress(dev)
    assert done == len(f) and error == 0 and rounds >= 1
    assert launches == 3 + rounds * dev.extra["launches_per_round"]
    # a budget-limited solve still ends: the round budget bounds the device loop
    cut = solve_batched(med, f[:2], th[:2], tolerance=1e-12, max_iterations=5)
    torch.cuda.synchronize()
    assert cut.reasons() == ["iteration_budget"] * 2
