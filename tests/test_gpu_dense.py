"""The dense (8th-order staggered, split-PML) operator on the GPU against the
reference's own output (golden) and the FFT-evaluated oracle."""
import json

import numpy as np
import pytest
import torch

from conftest import GOLDEN, rel
from oracle import dense_ref as D

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN / "reference_dense.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 3e-6)])
def test_dense_operator_matches_reference(cuda, gold, dtype, tol):
    from nsrno_b200.dense import DenseGeometry, DenseSystem
    spec = json.loads(str(gold["spec"]))
    g = DenseGeometry(spec)
    prng = np.random.default_rng(int(gold["probe_seed"]))
    p = prng.standard_normal((g.H, g.W)) + 1j * prng.standard_normal((g.H, g.W))
    pt = torch.as_tensor(p, device=cuda).to(dtype)
    inner = (slice(g.pz, g.pz + g.h), slice(g.px, g.px + g.w))
    for k, f in enumerate(gold["freqs"]):
        s = DenseSystem(g, gold["medium"], gold["alpha"], f, device=cuda)
        y = s.apply(pt).cpu().numpy()
        yh = s.adjoint(pt).cpu().numpy()
        assert rel(y[inner], gold[f"y{k}"]) < tol
        assert rel(yh[inner], gold[f"yh{k}"]) < tol
        out = np.ones((g.H, g.W), bool)
        out[inner] = False
        assert np.array_equal(y[out], pt.cpu().numpy()[out])


def test_dense_operator_matches_oracle_on_a_larger_grid(cuda):
    from nsrno_b200.dense import DenseGeometry, DenseSystem
    spec = {"medium_shape": [96, 128], "dx_m": 5e-5, "x0_m": -0.003, "z0_m": -0.0002, "native_dt_s": 2.5e-9,
            "pml": 12, "eta_per_unit_alpha": [0.012, 0.021], "taus_s": [2.0e-8, 1.5e-7],
            "source_c_lookup_zx": [10, 20]}
    rng = np.random.default_rng(8)
    medium = np.stack((1500 + 70 * rng.standard_normal((96, 128)), 1000 + 40 * rng.standard_normal((96, 128))))
    alpha = rng.uniform(0.1, 1.0, (96, 128))
    g = DenseGeometry(spec)
    og = D.DenseGeometry(spec)
    p = rng.standard_normal((2, g.H, g.W)) + 1j * rng.standard_normal((2, g.H, g.W))
    q = rng.standard_normal((2, g.H, g.W)) + 1j * rng.standard_normal((2, g.H, g.W))
    for f in (4.2e6, 8.8e6):
        s = DenseSystem(g, medium, alpha, f, device=cuda)
        o = D.DenseSystem(og, medium, alpha, f)
        y = s.apply(torch.as_tensor(p, device=cuda)).cpu().numpy()
        yh = s.adjoint(torch.as_tensor(p, device=cuda)).cpu().numpy()
        for k in range(2):
            assert rel(y[k], o.apply(p[k])) < 1e-12
            assert rel(yh[k], o.adjoint(p[k])) < 1e-12
        # adjoint identity on the device
        qy = np.vdot(q, y)
        aq = np.vdot(s.adjoint(torch.as_tensor(q, device=cuda)).cpu().numpy(), p)
        assert abs(qy - aq) / abs(qy) < 1e-12
