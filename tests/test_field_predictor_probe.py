"""Why the learned part is a preconditioner and not a field predictor (CPU).

A network that predicts the wavefield (the 4-level U-Net of the learned
warm-start configuration) helps Krylov only through the relative residual of
its prediction.  On a breast-like medium at the band's high end, a prediction
whose field error is a smooth 6% (already a very good predictor) still leaves
a relative residual of 0.03: the discrete Helmholtz operator amplifies any
field error by its wavenumber contrast.  BiCGSTAB from such a start saves
about 1.5 of the six decades of a 1e-6 solve (a quarter of the iterations if
convergence were linear), whereas the learned preconditioner shortens every
decade (about 3x fewer iterations on the benchmark medium).  This is the measured basis for building the reference's
learned preconditioner (nsrno/conditioned_wave.py:94-117) and not a field
predictor.
"""
import numpy as np

from conftest import spec_of
from oracle import helmholtz_ref as H


def test_a_six_percent_field_error_leaves_a_large_residual():
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=7, nz=128, nx=192, n_pml=16, n_rx=40, rx_pitch=4, bins=[8.2e6], n_angles=1)
    spec = spec_of(rec)
    f, th = rec.systems()
    A = H.operator(spec, rec.c, rec.rho, rec.alpha, f[0])
    b = H.plane_wave_rhs(spec, f[0], th[0])
    u = H.solve_lu(A, b)
    rng = np.random.default_rng(0)
    # a smooth multiplicative error field (correlation length of a few wavelengths)
    zz, xx = np.meshgrid(np.arange(rec.nz), np.arange(rec.nx), indexing="ij")
    smooth = np.zeros((rec.nz, rec.nx), complex)
    for _ in range(12):
        cz, cx = rng.uniform(0, rec.nz), rng.uniform(0, rec.nx)
        smooth += (rng.standard_normal() + 1j * rng.standard_normal()) * \
            np.exp(-((zz - cz) ** 2 + (xx - cx) ** 2) / (2 * 14.0 ** 2))
    err = smooth.ravel() * u
    err *= 0.06 * np.linalg.norm(u) / np.linalg.norm(err)
    guess = u + err
    field_error = np.linalg.norm(guess - u) / np.linalg.norm(u)
    residual = H.relative_residual(A, guess, b)
    assert abs(field_error - 0.06) < 1e-12
    # the start is worth at most about 1.7 of the six decades of a 1e-6 solve
    assert residual > 0.02, residual
