"""CPU checks of the host-side logic: synthetic records and API contracts that
are decided before any device work."""
import numpy as np
import pytest
import torch


def test_blob_record_is_seeded_and_vanishes_in_pml():
    from nsrno_b200.media import blob_record
    a, b = blob_record(), blob_record()
    assert np.array_equal(a.c, b.c) and np.array_equal(a.rho, b.rho)
    assert a.c.shape == (256, 256) and a.h == 1e-4 and a.n_pml == 20
    pml = ~a.interior()
    assert np.all(a.c[pml] == 1500.0) and np.all(a.rho[pml] == 1000.0)
    assert 1390 < a.c.min() <= 1500 <= a.c.max() < 1610
    assert len(a.rx_cols) == 192 and np.all(np.diff(a.rx_cols) == 1)
    f, th = a.systems()
    assert len(f) == 6 and set(np.round(np.rad2deg(th))) == {-15.0, 0.0, 15.0}


def test_breast_record_matches_its_description():
    from nsrno_b200.media import breast_bins, breast_record
    r = breast_record()
    assert (r.nz, r.nx, r.h) == (768, 1024, 5e-5)
    bins = breast_bins()
    assert len(bins) == 294 and abs(bins[0] - 4.015e6) < 1e3 and abs(bins[-1] - 8.896e6) < 1e3
    assert len(r.angles) == 11 and abs(np.rad2deg(r.angles[0]) + 25) < 1e-9
    f, th = r.systems()
    assert len(f) == 3234
    assert 1419 <= r.c.min() and r.c.max() <= 1561
    assert 919 <= r.rho.min() and r.rho.max() <= 1061
    assert np.all(r.c[~r.interior()] == 1500.0)
    assert np.all(r.rx_cols >= 0) and np.all(r.rx_cols < r.nx) and np.all(np.diff(r.rx_cols) == 4)
    # coupling layer under the array is water with alpha 0.002
    rows = slice(r.face, r.face + 20)
    assert np.all(r.c[rows] == 1500.0) and np.allclose(r.alpha[rows], 0.002)


def test_solve_frequency_contract_errors():
    from nsrno_b200 import Geometry, PlaneWaveModel, solve_frequency
    geo = Geometry(nz=64, nx=64, h=1e-4, n_pml=8, face=10, rx_cols=np.arange(10, 50), aperture_half_width=2e-3)
    model = PlaneWaveModel(geo, [0.0])
    medium = torch.zeros(1, 2, 64, 64, requires_grad=True)
    with pytest.raises(ValueError, match="implicit-adjoint"):
        solve_frequency(model, medium, 1e6, 0)
    with pytest.raises(ValueError, match="multiple of restart"):
        solve_frequency(model, medium.detach(), 1e6, 0, max_iterations=100, restart=32)


def test_surrogate_rejects_bins_outside_band():
    from nsrno_b200 import Geometry, HelmholtzSurrogate, bin_frequency
    geo = Geometry(nz=64, nx=64, h=1e-4, n_pml=8, face=10, rx_cols=np.arange(10, 50), aperture_half_width=2e-3)
    s = HelmholtzSurrogate(geo, [0.0], device="cpu")
    with pytest.raises(ValueError, match="outside cached dense band"):
        s(torch.zeros(2, 64, 64), torch.zeros(64, 64), 100)
    assert abs(bin_frequency(360) - 360 * 40e6 / 2401) < 1e-6


def test_medium_requires_cuda_tensors_without_a_gpu():
    from nsrno_b200 import Geometry, Medium
    geo = Geometry(nz=16, nx=16, h=1e-4, n_pml=2, face=3, rx_cols=np.arange(4), aperture_half_width=1e-3)
    if torch.cuda.is_available():
        pytest.skip("device present")
    with pytest.raises((ValueError, RuntimeError)):
        Medium(geo, np.full((16, 16), 1500.0), np.full((16, 16), 1000.0), np.zeros((16, 16)), device="cpu")


def test_receiver_response_is_band_limited():
    from nsrno_b200 import receiver_response
    mid = receiver_response(5.8e6)
    assert 0.5 < mid <= 1.01
    assert receiver_response(1.0e6) < 1e-3
    assert receiver_response(15e6) < 1e-3


def test_gauss_newton_accepts_only_near_tolerance_stalls():
    """The step's convergence check: converged systems pass; a system that
    used its iteration budget passes only within accept_factor x tolerance
    (and is counted); anything else, or a non-finite residual, raises."""
    from types import SimpleNamespace
    from nsrno_b200 import _lib
    from nsrno_b200.gauss_newton import _require_converged

    def res(status, resid):
        st = torch.as_tensor(status, dtype=torch.int32)
        return SimpleNamespace(status=st, residual=torch.as_tensor(resid, dtype=torch.float64),
                               reasons=lambda: [_lib.REASONS[int(s)] for s in st])

    C, B, D = _lib.CONVERGED, _lib.ITERATION_BUDGET, _lib.DIVERGED
    assert _require_converged(res([C, C], [1e-7, 9e-7]), "forward", 1e-6, 2.0) == 0
    assert _require_converged(res([C, B, B], [1e-7, 1.1e-6, 2e-6]), "adjoint", 1e-6, 2.0) == 2
    with pytest.raises(RuntimeError):
        _require_converged(res([C, B], [1e-7, 2.5e-6]), "adjoint", 1e-6, 2.0)
    with pytest.raises(RuntimeError):
        _require_converged(res([B], [float("nan")]), "adjoint", 1e-6, 2.0)
    with pytest.raises(RuntimeError):
        _require_converged(res([D], [1e-7]), "adjoint", 1e-6, 2.0)
    with pytest.raises(RuntimeError):   # strict without a tolerance
        _require_converged(res([B], [1e-7]), "observed data")
