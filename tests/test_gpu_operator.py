"""GPU parity of the stand-alone operators against the CPU oracle."""
import math

import numpy as np
import pytest
import torch

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu


def small_record(nz=48, nx=64, n_pml=6, seed=5):
    from nsrno_b200.media import Record
    rng = np.random.default_rng(seed)
    c = 1500 + 80 * rng.standard_normal((nz, nx))
    rho = 1000 + 60 * rng.standard_normal((nz, nx))
    alpha = rng.uniform(0.0, 1.5, (nz, nx))
    return Record(nz=nz, nx=nx, h=1e-4, n_pml=n_pml, face=n_pml + 2, rx_cols=np.arange(8, nx - 8, 2),
                  aperture_half_width=(nx - 20) * 1e-4 / 2, c=c.astype(np.float32), rho=rho.astype(np.float32),
                  alpha=alpha.astype(np.float32), frequencies=np.array([1.0e6, 2.3e6]), angles=np.array([0.0, 0.2]))


def medium_of(rec, dev):
    from nsrno_b200 import Geometry, Medium
    return Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=dev)


def planes(med):
    a, b, t = med.coef64.cpu().numpy()
    return a, b, t


def test_material_planes_match_rounded_double(cuda):
    rec = small_record()
    med = medium_of(rec, cuda)
    a, b, t = H.material(spec_of(rec), rec.c, rec.rho, rec.alpha)
    ga, gb, gt = med.coef.cpu().numpy()
    for ref, got in ((a, ga), (b, gb), (t, gt)):
        ulps = np.abs(ref.astype(np.float32).view(np.int32) - got.view(np.int32))
        assert ulps.max() <= 1
    da, db, dt = med.coef64.cpu().numpy()
    for ref, got in ((a, da), (b, db), (t, dt)):
        assert np.max(np.abs(ref - got) / np.maximum(np.abs(ref), 1e-300)) < 1e-15


@pytest.mark.parametrize("adjoint", [False, True])
def test_apply_matches_oracle(cuda, adjoint):
    from nsrno_b200 import apply
    rec = small_record()
    spec = spec_of(rec)
    med = medium_of(rec, cuda)
    a, b, t = planes(med)
    rng = np.random.default_rng(1)
    S = len(rec.frequencies)
    x = rng.standard_normal((S, rec.nz, rec.nx)) + 1j * rng.standard_normal((S, rec.nz, rec.nx))
    y64 = apply(med, torch.as_tensor(x, device=cuda), rec.frequencies, adjoint=adjoint).cpu().numpy()
    y32 = apply(med, torch.as_tensor(x.astype(np.complex64), device=cuda), rec.frequencies,
                adjoint=adjoint).cpu().numpy()
    for s, f in enumerate(rec.frequencies):
        A = H.operator_planes(spec, a, b, t, f)
        if adjoint:
            A = A.conj().T.tocsr()
        ref = (A @ x[s].ravel()) * rec.h ** 2
        assert rel(y64[s].ravel(), ref) < 1e-13
        assert rel(y32[s].ravel(), ref) < 2e-6


def test_operator_is_complex_symmetric(cuda):
    from nsrno_b200 import apply
    rec = small_record()
    med = medium_of(rec, cuda)
    rng = np.random.default_rng(2)
    x = torch.as_tensor(rng.standard_normal((1, rec.nz, rec.nx)) + 1j * rng.standard_normal((1, rec.nz, rec.nx)),
                        device=cuda)
    y = torch.as_tensor(rng.standard_normal((1, rec.nz, rec.nx)) + 1j * rng.standard_normal((1, rec.nz, rec.nx)),
                        device=cuda)
    f = [1.7e6]
    left = (y * apply(med, x, f)).sum()
    right = (apply(med, y, f) * x).sum()
    assert abs(left - right) / abs(left) < 1e-13
    # adjoint identity <y, A x> = <A^H y, x>
    l2 = (y.conj() * apply(med, x, f)).sum()
    r2 = (apply(med, y, f, adjoint=True).conj() * x).sum()
    assert abs(l2 - r2) / abs(l2) < 1e-13


def numpy_precondition(x, nz, nx, kh2, shift, adjoint=False):
    qz = np.sin(np.pi * np.arange(nz) / nz) ** 2
    qx = np.sin(np.pi * np.arange(nx) / nx) ** 2
    sym = -4.0 * (qz[:, None] + qx[None, :]) + kh2 * (1 + 1j * shift)
    mul = 1.0 / sym
    if adjoint:
        mul = mul.conj()
    return np.fft.ifft2(np.fft.fft2(x) * mul)


@pytest.mark.parametrize("shape", [(48, 64), (81, 81), (162, 96), (256, 256), (768, 1024), (24, 2048),
                                   (110, 140), (961, 122), (1056, 1216)])
@pytest.mark.parametrize("adjoint", [False, True])
def test_precondition_matches_numpy_fft(cuda, shape, adjoint):
    from nsrno_b200 import precondition
    nz, nx = shape
    rec = small_record(nz=nz, nx=nx, n_pml=4)
    med = medium_of(rec, cuda)
    rng = np.random.default_rng(3)
    freqs = np.array([1.1e6, 3.0e6])
    x = (rng.standard_normal((2, nz, nx)) + 1j * rng.standard_normal((2, nz, nx))).astype(np.complex64)
    y = precondition(med, torch.as_tensor(x, device=cuda), freqs, shift=0.15, adjoint=adjoint).cpu().numpy()
    for s, f in enumerate(freqs):
        kh2 = (2 * math.pi * f / rec.c0 * rec.h) ** 2
        ref = numpy_precondition(x[s].astype(np.complex128), nz, nx, kh2, 0.15, adjoint)
        assert rel(y[s], ref) < 3e-6


def test_plane_wave_rhs_matches_oracle(cuda):
    from nsrno_b200 import plane_wave_rhs
    rec = small_record()
    spec = spec_of(rec)
    med = medium_of(rec, cuda)
    b = plane_wave_rhs(med, rec.frequencies, rec.angles).cpu().numpy()
    for s, (f, th) in enumerate(zip(rec.frequencies, rec.angles)):
        assert rel(b[s].ravel(), H.plane_wave_rhs(spec, f, th)) < 1e-14


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_grad_accum_matches_oracle(cuda, dtype):
    from nsrno_b200 import grad_accum
    rec = small_record()
    spec = spec_of(rec)
    med = medium_of(rec, cuda)
    a, b, t = planes(med)
    rng = np.random.default_rng(4)
    S = 2
    u = (rng.standard_normal((S, rec.nz, rec.nx)) + 1j * rng.standard_normal((S, rec.nz, rec.nx))).astype(dtype)
    lam = (rng.standard_normal((S, rec.nz, rec.nx)) + 1j * rng.standard_normal((S, rec.nz, rec.nx))).astype(dtype)
    gc, gr = grad_accum(med, rec.frequencies, torch.as_tensor(u, device=cuda), torch.as_tensor(lam, device=cuda))
    ref_c = np.zeros((rec.nz, rec.nx))
    ref_r = np.zeros((rec.nz, rec.nx))
    for s, f in enumerate(rec.frequencies):
        c_, r_ = H.material_gradient_planes(spec, a, b, t, f, u[s], lam[s])
        ref_c += c_
        ref_r += r_
    assert rel(gc.cpu().numpy(), ref_c) < 1e-12
    assert rel(gr.cpu().numpy(), ref_r) < 1e-12


def test_band_rf_matches_irfft(cuda):
    """predict_band_rf (nsrno/wave_operator.py:169-180): irfft(n=2401, norm='forward')
    of a spectrum that is zero except on the given bins."""
    from nsrno_b200 import band_rf
    rng = np.random.default_rng(4)
    bins = np.array([241, 300, 377, 534, 1000])
    spec = rng.standard_normal((6, bins.size)) + 1j * rng.standard_normal((6, bins.size))
    full = np.zeros((6, 1201), complex)
    full[:, bins] = spec
    want = np.fft.irfft(full, n=2401, axis=-1, norm="forward")
    got = band_rf(torch.as_tensor(spec, device=cuda), bins).cpu().numpy()
    assert rel(got, want) < 1e-12
    with pytest.raises(ValueError, match="Positive RF bin out of range"):
        band_rf(torch.as_tensor(spec, device=cuda), np.array([0, 300, 377, 534, 1000]))


def test_true_residual_matches_oracle(cuda):
    """nsr_true_residual against the oracle's relative residual, plane-wave and given rhs, forward and adjoint."""
    from nsrno_b200 import Geometry, Medium, true_residual
    from nsrno_b200.media import blob_record
    rec = blob_record(nz=48, nx=64, n_pml=6, h=2e-4, n_blobs=2, frequencies=(0.8e6,), n_rx=16)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, rec.nz, rec.nx)) + 1j * rng.standard_normal((2, rec.nz, rec.nx))
    f = [0.8e6, 0.8e6]
    th = [0.1, -0.2]
    got = true_residual(med, torch.as_tensor(x, device=cuda), f, th).cpu().numpy()
    A = H.operator_planes(spec, a, b, t, 0.8e6)
    for s in range(2):
        want = H.relative_residual(A, x[s].ravel(), H.plane_wave_rhs(spec, f[s], th[s]))
        assert abs(got[s] - want) < 1e-12 * want
    rhs = rng.standard_normal((2, rec.nz, rec.nx)) + 1j * rng.standard_normal((2, rec.nz, rec.nx))
    got = true_residual(med, torch.as_tensor(x, device=cuda), f, rhs=torch.as_tensor(rhs, device=cuda),
                        adjoint=True).cpu().numpy()
    AH = A.conj().T.tocsr()
    for s in range(2):
        want = H.relative_residual(AH, x[s].ravel(), rhs[s].ravel())
        assert abs(got[s] - want) < 1e-12 * want
