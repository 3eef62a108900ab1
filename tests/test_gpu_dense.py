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


def dense_case(gold, cuda):
    from nsrno_b200.dense import DenseGeometry, DenseSystem
    g = DenseGeometry(json.loads(str(gold["spec"])))
    return g, DenseSystem(g, gold["medium"], gold["alpha"], float(gold["freqs"][0]), device=cuda)


@pytest.mark.parametrize("adjoint", [False, True])
def test_dense_preconditioner_matches_reference(cuda, gold, adjoint):
    g, s = dense_case(gold, cuda)
    prng = np.random.default_rng(int(gold["probe_seed"]))
    p = prng.standard_normal((g.H, g.W)) + 1j * prng.standard_normal((g.H, g.W))
    y = s.fixed_preconditioner(adjoint=adjoint)(torch.as_tensor(p, device=cuda)).cpu().numpy()
    if adjoint:
        o = D.DenseSystem(D.DenseGeometry(json.loads(str(gold["spec"]))), gold["medium"], gold["alpha"],
                          float(gold["freqs"][0]))
        assert rel(y, o.fixed_preconditioner(p, adjoint=True)) < 2e-5
    else:
        assert rel(y, gold["precondition"]) < 2e-5


def test_dense_assembly_matches_reference(cuda, gold):
    """S(src) - S0(src) - A p_ref + A0 p_ref (nsrno/dense_wave.py:46-57) on the device."""
    from nsrno_b200.dense import assemble, homogeneous_system
    g, s = dense_case(gold, cuda)
    s0 = homogeneous_system(g, float(gold["freqs"][0]), device=cuda)
    line = torch.as_tensor(gold["assembly_line"], device=cuda)
    pref = torch.as_tensor(gold["assembly_pref"], device=cuda)
    rhs = assemble(s, s0, line, pref).cpu().numpy()
    assert rel(rhs, gold["assembly_rhs"]) < 1e-12
    assert rel(s.source(line).cpu().numpy(), gold["source"]) < 1e-12


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-7), (torch.complex64, 1e-4)])
def test_dense_gmres_solve_matches_reference(cuda, gold, dtype, tol):
    """GMRES(32) with the fixed preconditioner on the dense operator against the
    reference's own converged solve (nsrno/wave_solver.py:9-36)."""
    from nsrno_b200.dense import solve
    g, s = dense_case(gold, cuda)
    b = torch.as_tensor(gold["solve_rhs"], device=cuda).to(dtype)
    x, info = solve(s, b, tolerance=1e-9 if dtype == torch.complex128 else 1e-5, max_cycles=200)
    assert info["reason"] == "converged"
    assert rel(x.cpu().numpy(), gold["solve_x"]) < tol


def test_dense_adjoint_solve(cuda, gold):
    from nsrno_b200.dense import solve
    g, s = dense_case(gold, cuda)
    b = torch.as_tensor(gold["solve_rhs"], device=cuda)
    x, info = solve(s, b, adjoint=True, tolerance=1e-9, max_cycles=200)
    assert info["reason"] == "converged"
    r = s.adjoint(x) - b
    assert float(r.norm() / b.norm()) < 1e-9


def test_homogeneous_reference_fields(cuda, gold, tmp_path):
    """Uniform-medium reference fields in the on-disk layout reference/a{angle:02d}.npy
    [bins, h, w] (nsrno/dense_wave.py:39-41, scripts/prepare_wave_teachers.py:22-35)."""
    from nsrno_b200.dense import DenseGeometry, homogeneous_reference, save_reference
    g = DenseGeometry(json.loads(str(gold["spec"])))
    freqs = [float(f) for f in gold["freqs"]]
    lines = np.broadcast_to(gold["assembly_line"], (2,) + gold["assembly_line"].shape).copy()
    fields = homogeneous_reference(g, freqs, lines, tolerance=1e-6, device=cuda)
    assert fields.shape == (2, 2, g.h, g.w) and fields.dtype == torch.complex64
    og = D.DenseGeometry(json.loads(str(gold["spec"])))
    for k, f in enumerate(freqs):
        s0 = D.homogeneous(og, f)
        src = s0.source(lines[k])
        for a in range(2):
            p = np.zeros((og.H, og.W), complex)
            p[og.pz:og.pz + og.h, og.px:og.px + og.w] = fields[a, k].cpu().numpy()
            assert rel(s0.apply(p), src[a]) < 1e-5
    save_reference(tmp_path, fields)
    assert np.load(tmp_path / "a01.npy").shape == (2, g.h, g.w)


def _spec(h, w):
    return {"medium_shape": [h, w], "dx_m": 5e-5, "x0_m": -0.004, "z0_m": -0.0002, "native_dt_s": 2.5e-9,
            "pml": 12, "eta_per_unit_alpha": [0.012, 0.021], "taus_s": [2.0e-8, 1.5e-7],
            "source_c_lookup_zx": [10, 20]}


def _medium(h, w, seed):
    rng = np.random.default_rng(seed)
    medium = np.stack((1500 + 40 * rng.standard_normal((h, w)), 1000 + 30 * rng.standard_normal((h, w))))
    return medium, rng.uniform(0.1, 1.0, (h, w))


def test_dense_preconditioner_at_the_reference_padding(cuda):
    """The reference pads its 961 x 1121 medium to 1056 x 1216 = (2^5 3 11) x (2^6 19)
    (nsrno/conditioned_wave.py:16-22); the preconditioner runs at that size."""
    from nsrno_b200.dense import DenseGeometry, DenseSystem
    spec = _spec(961, 1121)
    g = DenseGeometry(spec)
    assert (g.H, g.W) == (1056, 1216)
    medium, alpha = _medium(961, 1121, 3)
    s = DenseSystem(g, medium, alpha, 6.2e6, device=cuda)
    o = D.DenseSystem(D.DenseGeometry(spec), medium, alpha, 6.2e6)
    rng = np.random.default_rng(4)
    p = rng.standard_normal((g.H, g.W)) + 1j * rng.standard_normal((g.H, g.W))
    for adjoint in (False, True):
        y = s.fixed_preconditioner(adjoint=adjoint)(torch.as_tensor(p, device=cuda)).cpu().numpy()
        assert rel(y, o.fixed_preconditioner(p, adjoint=adjoint)) < 2e-5


@pytest.mark.parametrize("adjoint", [False, True])
def test_dense_device_solve_on_a_prime_padding(cuda, adjoint):
    """80 x 150 pads to 160 x 224 = (2^5 5) x (2^5 7): GMRES(24) on the device
    for three fields as one vector; the FP64 residual of every field, checked
    with the oracle operator, meets the tolerance."""
    from nsrno_b200.dense import DenseGeometry, DenseSystem, solve
    spec = _spec(80, 150)
    g = DenseGeometry(spec)
    assert (g.H, g.W) == (160, 224)
    medium, alpha = _medium(80, 150, 5)
    s = DenseSystem(g, medium, alpha, 5.1e6, device=cuda)
    o = D.DenseSystem(D.DenseGeometry(spec), medium, alpha, 5.1e6)
    rng = np.random.default_rng(6)
    b = (rng.standard_normal((3, g.H, g.W)) + 1j * rng.standard_normal((3, g.H, g.W))) * o.g.mask
    x, info = solve(s, torch.as_tensor(b, device=cuda), adjoint=adjoint, tolerance=1e-8, max_cycles=400)
    assert info["reason"] == "converged" and info["residual"] < 1e-8
    assert info["max_angle_residual"] < 1e-7
    x = x.cpu().numpy()
    for k in range(3):
        ax = o.adjoint(x[k]) if adjoint else o.apply(x[k])
        assert rel(ax, b[k]) < 1e-7


def test_dense_implicit_gradient_matches_reference_autograd(cuda, gold):
    """d/d(c, rho) of -Re sum conj(lam) mask (A(m)(mask (u + pref)) - S(m) line), the
    scalar ImplicitChannels.backward differentiates (nsrno/dense_wave.py:250-255):
    the device contraction plus the chain rule through the coefficient planes
    against the reference's own autograd (golden), for seeded fields."""
    from nsrno_b200.dense import material_gradient
    g, s = dense_case(gold, cuda)
    u = torch.as_tensor(gold["grad_u"], device=cuda)
    pref = torch.as_tensor(gold["assembly_pref"], device=cuda)
    lam = torch.as_tensor(gold["grad_lam"], device=cuda)
    line = torch.as_tensor(gold["assembly_line"], device=cuda)
    grad = material_gradient(s, torch.as_tensor(gold["medium"]), torch.as_tensor(gold["alpha"]), u + pref, lam, line)
    assert rel(grad.cpu().numpy(), gold["grad_medium"]) < 1e-10


def test_dense_surrogate_forward_backward(cuda):
    """The dense drop-in of DenseSurrogate: converged channels equal those of
    the oracle operator's own converged solve, and the implicit gradient
    agrees with central differences of the GPU forward along a smooth
    direction (1e-4)."""
    from nsrno_b200.dense import DenseAcquisition, DenseGeometry, DenseSurrogate
    from oracle import helmholtz_ref as H
    spec = _spec(40, 52)
    spec.update(x0_m=-0.0013, rx_count=12, rx_pitch_m=0.0002, rx_first_m=-0.0011)
    g = DenseGeometry(spec)
    medium, alpha = _medium(40, 52, 11)
    rng = np.random.default_rng(12)
    lines = rng.standard_normal((1, 2, 52)) + 1j * rng.standard_normal((1, 2, 52))
    data = DenseAcquisition(g, [300], lines, device=cuda, tolerance=1e-10)
    sur = DenseSurrogate(data)
    m = torch.as_tensor(medium, device=cuda).requires_grad_(True)
    a = torch.as_tensor(alpha, device=cuda)
    out = sur(m, a, 300, tolerance=1e-10)
    assert out.shape == (2, 12)
    # oracle: the same assembled right-hand side solved by the oracle operator
    o = D.DenseSystem(D.DenseGeometry(spec), medium, alpha, DenseAcquisition.frequency(300))
    o0 = D.homogeneous(D.DenseGeometry(spec), DenseAcquisition.frequency(300))
    pref = data.reference(300, [0, 1]).cpu().numpy()
    rhs = D.assemble(o, o0, lines[0], pref)
    for k in range(2):
        x, reason, _ = H.gmres(lambda v: o.apply(v.reshape(g.H, g.W)).ravel(), rhs[k].ravel(), restart=48,
                               max_cycles=400, tolerance=1e-11,
                               precondition=lambda v: o.fixed_preconditioner(v.reshape(g.H, g.W)).ravel())
        assert reason == "converged"
        ch = x.reshape(g.H, g.W)[g.face, g.rx_cols]
        from nsrno_b200.solver import receiver_response
        assert rel(out[k].detach().cpu().numpy(), ch * receiver_response(DenseAcquisition.frequency(300))) < 1e-6
    target = out.detach() * 0.9
    loss = 0.5 * (out - target).abs().square().sum()
    loss.backward()
    grad = m.grad.detach()
    xx, zz = np.meshgrid(np.arange(52), np.arange(40))
    win = torch.as_tensor(np.exp(-((xx - 26) ** 2 + (zz - 22) ** 2) / (2 * 5.0 ** 2)), device=cuda)
    d = torch.stack((win * 3.0, win * -2.0))

    def misfit(h):
        with torch.no_grad():
            o2 = sur(torch.as_tensor(medium, device=cuda) + h * d, a, 300, tolerance=1e-11)
            return float(0.5 * (o2 - target).abs().square().sum())
    fd = (misfit(1e-3) - misfit(-1e-3)) / 2e-3
    analytic = float((grad * d).sum())
    assert abs(analytic - fd) < 1e-4 * abs(analytic), (analytic, fd)
