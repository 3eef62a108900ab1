"""The CPU oracle pinned against the reference's golden vectors and known answers."""
import math

import numpy as np
import pytest
from scipy import sparse
from scipy.special import hankel1

from conftest import rel
from oracle import helmholtz_ref as H


def fixture_spec(golden):
    axis = golden["fixture_axis_mm"]
    h = float(axis[1] - axis[0]) * 1e-3
    n = axis.size
    return H.Spec(nz=n, nx=n, h=h, n_pml=int(round(float(golden["fixture_pml_mm"]) * 1e-3 / h)),
                  c0=float(golden["fixture_c0"]))


def fixture_weights(golden, n):
    return sparse.csc_matrix((golden["weights_val"], (golden["weights_row"], golden["weights_col"])),
                             shape=(n, 4))


def test_matrix_matches_reference_solver_matrix(golden):
    nz, nx = (int(v) for v in golden["matrix_shape"])
    spec = H.Spec(nz=nz, nx=nx, h=float(golden["matrix_h_mm"]) * 1e-3, n_pml=int(golden["matrix_pml"]),
                  c0=float(golden["matrix_c0"]))
    a = 1.0 + golden["matrix_me"]
    b = 1.0 + golden["matrix_mk"]
    ours = H.operator_planes(spec, a, b, np.zeros_like(a), float(golden["matrix_freq_mhz"]) * 1e6)
    ref = sparse.coo_matrix((golden["matrix_val"], (golden["matrix_row"], golden["matrix_col"])),
                            shape=ours.shape).tocsr()
    diff = abs(ours - ref).max()
    assert diff <= 1e-14 * abs(ref).max()
    assert ours.nnz == ref.nnz


def test_solve_matches_reference_fixture(golden):
    spec = fixture_spec(golden)
    W = fixture_weights(golden, spec.n)
    A = H.operator_planes(spec, np.ones((spec.nz, spec.nx)), np.ones((spec.nz, spec.nx)),
                          np.zeros((spec.nz, spec.nx)), float(golden["fixture_freq_mhz"]) * 1e6)
    u = H.solve_lu(A, -W.toarray() / spec.h ** 2)
    assert rel(u, golden["fields"]) < 1e-12
    assert rel(W.T @ u, golden["response"]) < 1e-12
    assert H.relative_residual(A, u[:, 0], -W.toarray()[:, 0] / spec.h ** 2) < 1e-12


def test_gradient_matches_reference_born_jacobian(golden):
    spec = fixture_spec(golden)
    n = spec.n
    W = fixture_weights(golden, n).toarray()
    f = float(golden["fixture_freq_mhz"]) * 1e6
    ones = np.ones((spec.nz, spec.nx))
    A = H.operator_planes(spec, ones, ones, 0 * ones, f)
    u = golden["fields"]
    r = golden["residual"].reshape(4, 4)
    lam = H.solve_lu(A.conj().T.tocsc(), W @ r.T)
    gc = np.zeros(n)
    gr = np.zeros(n)
    for k in range(4):
        c_, r_ = H.material_gradient_planes(spec, ones, ones, 0 * ones, f, u[:, k], lam[:, k])
        gc += c_.ravel()
        gr += r_.ravel()
    d_mk = -gc / 2.0
    d_me = -gr - d_mk
    ours = np.concatenate((golden["basis"].T @ d_mk, golden["basis"].T @ d_me))
    assert rel(ours, golden["gradient"]) < 1e-9


def test_green_function_and_refinement():
    """Known answer of tests/test_theranostic.py:141-158 on the oracle."""
    positions = np.array([[-3.2, 0.0], [3.2, 0.0], [0.0, 4.8]])
    d = np.linalg.norm(positions[:, None] - positions[None, :], axis=2) * 1e-3
    off = ~np.eye(3, dtype=bool)
    f = 0.15e6
    exact = 0.25j * hankel1(0, 2 * np.pi * f / 1540.0 * d[off])
    errors = []
    for intervals in (40, 80):
        n = intervals + 1
        h = 32.0 / intervals * 1e-3
        spec = H.Spec(nz=n, nx=n, h=h, n_pml=int(round(6e-3 / h)), c0=1540.0)
        idx = [int(round((p[1] + 16.0) * 1e-3 / h)) * n + int(round((p[0] + 16.0) * 1e-3 / h)) for p in positions]
        W = np.zeros((spec.n, 3))
        W[idx, range(3)] = 1.0
        ones = np.ones((n, n))
        A = H.operator_planes(spec, ones, ones, 0 * ones, f)
        u = H.solve_lu(A, -W / h ** 2)
        errors.append(rel((W.T @ u)[off], exact))
    assert errors[1] < 0.02
    assert errors[1] < 0.4 * errors[0]


def test_reciprocity_not_hermitian(golden):
    spec = fixture_spec(golden)
    W = fixture_weights(golden, spec.n).toarray()
    rng = np.random.default_rng(1)
    c = np.full((spec.nz, spec.nx), 1540.0)
    rho = np.full((spec.nz, spec.nx), 1000.0)
    inner = (slice(spec.n_pml + 2, spec.nz - spec.n_pml - 2),) * 2
    c[inner] += 40 * rng.standard_normal(c[inner].shape)
    rho[inner] += 30 * rng.standard_normal(c[inner].shape)
    A = H.operator(spec, c, rho, np.full_like(c, 0.5), 0.15e6)
    resp = W.T @ H.solve_lu(A, -W / spec.h ** 2)
    assert rel(resp, resp.T) < 1e-12
    assert np.linalg.norm(resp - resp.conj().T) > 1e-3 * np.linalg.norm(resp)


def test_attenuation_gradient_against_central_difference():
    """The c-dependence of the attenuation term enters d/dlog c (wave_operator.py:67)."""
    spec = H.Spec(nz=24, nx=28, h=1e-4, n_pml=4, face=6, rx_cols=np.arange(6, 22), aperture_half_width=8e-4)
    rng = np.random.default_rng(7)
    c = 1500 + 50 * rng.standard_normal((24, 28))
    rho = 1000 + 40 * rng.standard_normal((24, 28))
    alpha = rng.uniform(0.5, 2.0, (24, 28))
    f, th = 2.0e6, 0.1
    b = H.plane_wave_rhs(spec, f, th)
    d_obs = H.receivers(spec, H.solve_lu(H.operator(spec, c * 1.01, rho, alpha, f), b))

    def loss(cc, rr):
        r = H.receivers(spec, H.solve_lu(H.operator(spec, cc, rr, alpha, f), b)) - d_obs
        return 0.5 * float(np.vdot(r, r).real)

    A = H.operator(spec, c, rho, alpha, f)
    u = H.solve_lu(A, b)
    g = np.zeros(spec.n, complex)
    g[spec.face * spec.nx + spec.rx_cols] = H.receivers(spec, u) - d_obs
    lam = H.solve_lu(A.conj().T.tocsc(), g)
    gc, gr = H.material_gradient(spec, c, rho, alpha, f, u, lam)
    for (i, j) in [(10, 10), (15, 20), (5, 5)]:
        for which, grad in (("c", gc), ("r", gr)):
            eps = 1e-4
            cp, rp, cm, rm = c.copy(), rho.copy(), c.copy(), rho.copy()
            if which == "c":
                cp[i, j] *= math.exp(eps)
                cm[i, j] *= math.exp(-eps)
            else:
                rp[i, j] *= math.exp(eps)
                rm[i, j] *= math.exp(-eps)
            fd = (loss(cp, rp) - loss(cm, rm)) / (2 * eps)
            assert abs(fd - grad[i, j]) <= 1e-5 * abs(fd)


def test_krylov_ports_converge_to_lu():
    from nsrno_b200.media import blob_record
    rec = blob_record(nz=64, nx=64, n_pml=10, h=2e-4, n_blobs=2, frequencies=(0.6e6,))
    spec = H.Spec(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, face=rec.face, rx_cols=rec.rx_cols % rec.nx,
                  aperture_half_width=4e-3)
    A = H.operator(spec, rec.c, rec.rho, rec.alpha, 0.6e6)
    b = H.plane_wave_rhs(spec, 0.6e6, 0.2)
    ref = H.solve_lu(A, b)
    x, reason, steps = H.gmres(lambda v: A @ v, b, restart=30, max_cycles=400, tolerance=1e-9)
    assert reason == "converged"
    assert rel(x, ref) < 1e-6


def test_time_lu_frequency_reports_residual():
    from nsrno_b200.media import blob_record
    rec = blob_record(nz=64, nx=64, n_pml=10, h=2e-4, n_blobs=2)
    spec = H.Spec(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, face=rec.face, rx_cols=rec.rx_cols % rec.nx,
                  aperture_half_width=4e-3)
    fields, seconds, res = H.time_lu_frequency(spec, rec.c, rec.rho, rec.alpha, 1e6, rec.angles)
    assert fields.shape == (3, spec.n)
    assert res < 1e-10 and seconds > 0


def test_dense_oracle_matches_reference_operator():
    """The dense (8th-order, split-PML) operator and its adjoint against the reference's own output."""
    import json
    from conftest import GOLDEN
    from oracle import dense_ref as D
    with np.load(GOLDEN / "reference_dense.npz") as z:
        gold = {k: z[k] for k in z.files}
    spec = json.loads(str(gold["spec"]))
    g = D.DenseGeometry(spec)
    assert (g.H, g.W, g.pz, g.px) == (int(gold["H"]), int(gold["W"]), int(gold["pz"]), int(gold["px"]))
    prng = np.random.default_rng(int(gold["probe_seed"]))
    p = prng.standard_normal((g.H, g.W)) + 1j * prng.standard_normal((g.H, g.W))
    inner = (slice(g.pz, g.pz + g.h), slice(g.px, g.px + g.w))
    for k, f in enumerate(gold["freqs"]):
        s = D.DenseSystem(g, gold["medium"], gold["alpha"], f)
        assert rel(s.apply(p)[inner], gold[f"y{k}"]) < 1e-12
        assert rel(s.adjoint(p)[inner], gold[f"yh{k}"]) < 1e-12
        q = prng.standard_normal((g.H, g.W)) + 1j * prng.standard_normal((g.H, g.W))
        left = np.vdot(q, s.apply(p))
        right = np.vdot(s.adjoint(q), p)
        assert abs(left - right) / abs(left) < 1e-12


def test_operator_derivative_against_central_differences():
    """The directional derivative of the operator (the tangent / Born perturbation)."""
    spec = H.Spec(nz=20, nx=24, h=1e-4, n_pml=4, face=5, rx_cols=np.arange(4, 20), aperture_half_width=8e-4)
    rng = np.random.default_rng(11)
    c = 1500 + 40 * rng.standard_normal((20, 24))
    rho = 1000 + 30 * rng.standard_normal((20, 24))
    alpha = rng.uniform(0.3, 1.5, (20, 24))
    dc = rng.standard_normal((20, 24))
    dr = rng.standard_normal((20, 24))
    f = 2.5e6
    dA = H.operator_derivative(spec, c, rho, alpha, f, dc, dr)
    eps = 1e-5
    fd = (H.operator(spec, c * np.exp(eps * dc), rho * np.exp(eps * dr), alpha, f)
          - H.operator(spec, c * np.exp(-eps * dc), rho * np.exp(-eps * dr), alpha, f)) / (2 * eps)
    assert abs(dA - fd).max() <= 1e-7 * abs(fd).max()
    # tangent fields against central differences of the solve
    b = H.plane_wave_rhs(spec, f, 0.2)
    u = H.solve_lu(H.operator(spec, c, rho, alpha, f), b)
    du = H.born_fields(spec, c, rho, alpha, f, u, dc, dr)
    up = H.solve_lu(H.operator(spec, c * np.exp(eps * dc), rho * np.exp(eps * dr), alpha, f), b)
    um = H.solve_lu(H.operator(spec, c * np.exp(-eps * dc), rho * np.exp(-eps * dr), alpha, f), b)
    assert rel(du, (up - um) / (2 * eps)) < 1e-6


def test_dense_oracle_preconditioner_and_assembly_match_reference():
    """Fixed preconditioner, source and assembled right-hand side of the dense
    oracle against the reference's own output (complex128)."""
    import json
    from conftest import GOLDEN
    from oracle import dense_ref as D
    with np.load(GOLDEN / "reference_dense.npz") as z:
        gold = {k: z[k] for k in z.files}
    g = D.DenseGeometry(json.loads(str(gold["spec"])))
    prng = np.random.default_rng(int(gold["probe_seed"]))
    p = prng.standard_normal((g.H, g.W)) + 1j * prng.standard_normal((g.H, g.W))
    s = D.DenseSystem(g, gold["medium"], gold["alpha"], float(gold["freqs"][0]))
    assert rel(s.fixed_preconditioner(p), gold["precondition"]) < 1e-12
    assert rel(s.source(gold["assembly_line"]), gold["source"]) < 1e-12
    s0 = D.homogeneous(g, float(gold["freqs"][0]))
    rhs = D.assemble(s, s0, gold["assembly_line"], gold["assembly_pref"])
    assert rel(rhs, gold["assembly_rhs"]) < 1e-12
    x = gold["solve_x"][0]
    assert rel(s.apply(x), gold["solve_rhs"][0]) < 1e-9
