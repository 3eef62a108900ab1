"""GPU parity on the benchmarked configuration itself.

The throughput figures are quoted on the 1024 (x) x 768 (z) breast record at
0.05 mm: 11 angles (-25..+25 degrees) x 294 bins (4.015-8.896 MHz).  Its
highest bins have only 3.2 points per wavelength, the hardest systems of the
record.  Here the lowest and the highest bin, at both extreme angles, are
solved to a true relative residual of 1e-7 with the fixed and with the trained
learned preconditioner, and the fields and receiver IQ are compared with the
SuperLU solution of the same discretisation (theranostic/wave.py:240-273, one
factorisation per frequency shared by its angles).
"""
import numpy as np
import pytest
import torch
from scipy.sparse.linalg import splu

from conftest import rel, spec_of
from oracle import helmholtz_ref as H

pytestmark = pytest.mark.gpu

# field and IQ relative L2 against SuperLU at a true relative residual of 1e-7
TOL_FIELD = 1e-5


@pytest.fixture(scope="module")
def breast(cuda):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import breast_record
    rec = breast_record()
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    freqs = [float(rec.frequencies[0]), float(rec.frequencies[-1])]
    angles = [float(rec.angles[0]), float(rec.angles[-1])]
    spec = spec_of(rec)
    a, b, t = med.coef64.cpu().numpy()
    lu = {}
    for f in freqs:
        A = H.operator_planes(spec, a, b, t, f)
        factor = splu(A.tocsc())
        rhs = np.stack([H.plane_wave_rhs(spec, f, th) for th in angles], axis=1)
        x = factor.solve(rhs)
        assert max(H.relative_residual(A, x[:, k], rhs[:, k]) for k in range(len(angles))) < 1e-10
        lu[f] = x.T
    f_sys = np.repeat(freqs, len(angles))
    a_sys = np.tile(angles, len(freqs))
    return rec, med, spec, f_sys, a_sys, lu


@pytest.mark.parametrize("preconditioner", ["fixed", "learned"])
def test_benchmark_record_extreme_bins_match_lu(cuda, breast, preconditioner):
    from nsrno_b200 import solve_batched
    from nsrno_b200.learned import LearnedPreconditioner
    rec, med, spec, f_sys, a_sys, lu = breast
    setup = None
    if preconditioner == "learned":
        setup = LearnedPreconditioner.load(device=cuda).setup(med, np.unique(f_sys))
    res = solve_batched(med, f_sys, a_sys, tolerance=1e-7, max_iterations=8000, n_slots=len(f_sys),
                        return_fields=True, fields_dtype=torch.complex128, learned=setup)
    torch.cuda.synchronize()
    assert res.reasons() == ["converged"] * len(f_sys)
    assert float(res.residual.max()) < 1e-7
    fields = res.fields.cpu().numpy()
    iq = res.iq.cpu().numpy()
    n_angles = len(np.unique(a_sys))
    for s in range(len(f_sys)):
        ref = lu[float(f_sys[s])][s % n_angles]
        assert rel(fields[s].ravel(), ref) < TOL_FIELD, (s, rel(fields[s].ravel(), ref))
        assert rel(iq[s], H.receivers(spec, ref)) < TOL_FIELD, (s, rel(iq[s], H.receivers(spec, ref)))
