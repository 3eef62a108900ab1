"""GPU parity of the learned preconditioner: network and gains, apply and
adjoint, solves through it, the hand-written training gradient, and what the
trained network gains over the fixed preconditioner."""
import math

import numpy as np
import pytest
import torch

from conftest import GOLDEN, rel, spec_of
from oracle import helmholtz_ref as H
from oracle import learned_ref as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN / "reference_learned.npz") as z:
        return {k: z[k] for k in z.files}


def golden_medium(gold, dev):
    from nsrno_b200 import Geometry, Medium
    nz, nx = gold["c"].shape
    geo = Geometry(nz=nz, nx=nx, h=float(gold["h"]), n_pml=4, face=6, rx_cols=np.arange(8, 56),
                   aperture_half_width=1e-3, c0=float(gold["c0"]))
    return Medium(geo, gold["c"].astype(np.float32), gold["rho"].astype(np.float32),
                  gold["alpha"].astype(np.float32), device=dev)


def oracle_of(gold, med, params, f):
    return L.Learned(torch.as_tensor(params, dtype=torch.float64), med.c.double().cpu(), med.rho.double().cpu(),
                     med.alpha.double().cpu(), f, med.geometry.h, med.geometry.c0)


def test_setup_gains_match_oracle(cuda, gold):
    from nsrno_b200.learned import LearnedPreconditioner
    med = golden_medium(gold, cuda)
    freqs = [float(gold["frequency"]), 7.1e6]
    net = LearnedPreconditioner(gold["params"], device=cuda)
    st = net.setup(med, freqs)
    for k, f in enumerate(freqs):
        ref = oracle_of(gold, med, gold["params"], f)
        assert rel(st.gains[k, 0].cpu().numpy(), ref.inner.numpy()) < 1e-5
        assert rel(st.gains[k, 1].cpu().numpy(), ref.outer.numpy()) < 1e-5


@pytest.mark.parametrize("adjoint", [False, True])
def test_learned_apply_matches_oracle_and_reference(cuda, gold, adjoint):
    from nsrno_b200.learned import LearnedPreconditioner, learned_precondition
    med = golden_medium(gold, cuda)
    f = float(gold["frequency"])
    net = LearnedPreconditioner(gold["params"], device=cuda)
    st = net.setup(med, [f])
    probe = np.conj(gold["probe"])
    x = torch.as_tensor(probe[None].astype(np.complex64), device=cuda)
    y = learned_precondition(med, st, x, [f], adjoint=adjoint)[0].cpu().numpy()
    ref = oracle_of(gold, med, gold["params"], f)
    want = (ref.adjoint if adjoint else ref.apply)(torch.as_tensor(probe)).numpy()
    assert rel(y, want) < 2e-5
    # the reference module's own output, through the conjugate map of the 5-point path
    kh2 = (2 * math.pi * f / float(gold["c0"]) * float(gold["h"])) ** 2
    golden_out = gold["adjoint"] if adjoint else gold["apply"]
    assert rel(y, np.conj(golden_out) / kh2) < 2e-5


def test_untrained_network_equals_fixed_preconditioner(cuda, gold):
    from nsrno_b200 import precondition
    from nsrno_b200.learned import LearnedPreconditioner, learned_precondition
    med = golden_medium(gold, cuda)
    f = float(gold["frequency"])
    st = LearnedPreconditioner(device=cuda).setup(med, [f])
    x = torch.as_tensor(gold["probe"][None].astype(np.complex64), device=cuda)
    a = learned_precondition(med, st, x, [f]).cpu().numpy()
    b = precondition(med, x, [f]).cpu().numpy()
    assert rel(a, b) < 1e-6


def blob_case(dev):
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.media import blob_record
    rec = blob_record(nz=96, nx=128, n_pml=12, h=2e-4, n_blobs=3, frequencies=(0.9e6, 1.3e6))
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=dev)
    return rec, med


@pytest.mark.parametrize("adjoint", [False, True])
def test_solves_through_learned_preconditioner_match_lu(cuda, gold, adjoint):
    """BiCGSTAB and GMRES with non-trivial learned gains converge to the SuperLU solution."""
    from nsrno_b200 import gmres_batched, solve_batched
    from nsrno_b200.learned import LearnedPreconditioner
    rec, med = blob_case(cuda)
    spec = spec_of(rec)
    f, th = rec.systems()
    params = gold["params"].astype(np.float32) * 0.5
    params[8] = math.log(0.2)
    st = LearnedPreconditioner(params, device=cuda).setup(med, rec.frequencies)
    a, b, t = med.coef64.cpu().numpy()
    if adjoint:
        rng = np.random.default_rng(3)
        rhs = (rng.standard_normal((len(f), rec.nz, rec.nx)) + 1j * rng.standard_normal((len(f), rec.nz, rec.nx)))
        rhs_t = torch.as_tensor(rhs.astype(np.complex64), device=cuda)
        kw = dict(rhs=rhs_t, adjoint=True)
    else:
        kw = dict(angles=th)
    res_b = solve_batched(med, f, tolerance=1e-7, max_iterations=3000, return_fields=True, learned=st, n_slots=3, **kw)
    res_g = gmres_batched(med, f, tolerance=1e-7, max_iterations=3000, restart=30, return_fields=True, learned=st,
                          **kw)
    assert res_b.reasons() == ["converged"] * len(f)
    assert res_g.reasons() == ["converged"] * len(f)
    for s in range(len(f)):
        A = H.operator_planes(spec, a, b, t, f[s])
        if adjoint:
            ref = H.solve_lu(A.conj().T.tocsc(), rhs[s].astype(np.complex64).astype(np.complex128).ravel())
        else:
            ref = H.solve_lu(A, H.plane_wave_rhs(spec, f[s], th[s]))
        assert rel(res_b.fields[s].cpu().numpy().ravel(), ref) < 1e-5
        assert rel(res_g.fields[s].cpu().numpy().ravel(), ref) < 1e-5


@pytest.mark.parametrize("adjoint", [False, True])
def test_reused_slot_rebuilds_the_learned_multiplier(cuda, gold, adjoint):
    """One slot serving systems of alternating frequencies gives, system by
    system, exactly the iterations and receiver IQ of solving each system on
    its own: the slot's learned multiplier plane is rebuilt for every system
    it starts (a stale plane would only cost iterations, which is what this
    compares)."""
    from nsrno_b200 import solve_batched
    from nsrno_b200.learned import LearnedPreconditioner
    rec, med = blob_case(cuda)
    f, th = rec.systems()
    order = np.lexsort((f, th))          # consecutive systems alternate in frequency
    f, th = f[order], th[order]
    assert np.all(f[1:] != f[:-1])
    params = gold["params"].astype(np.float32) * 0.5
    params[8] = math.log(0.2)
    st = LearnedPreconditioner(params, device=cuda).setup(med, rec.frequencies)
    rng = np.random.default_rng(11)
    rhs = (rng.standard_normal((len(f), rec.nz, rec.nx)) + 1j * rng.standard_normal((len(f), rec.nz, rec.nx)))
    rhs = torch.as_tensor(rhs.astype(np.complex64), device=cuda)

    def run(sel):
        kw = dict(rhs=rhs[sel], adjoint=True) if adjoint else dict(angles=th[sel])
        return solve_batched(med, f[sel], tolerance=1e-7, max_iterations=3000, learned=st, n_slots=1, **kw)

    together = run(slice(None))
    assert together.reasons() == ["converged"] * len(f)
    for s in range(len(f)):
        alone = run(slice(s, s + 1))
        assert int(alone.iterations[0]) == int(together.iterations[s])
        assert torch.equal(alone.iq[0], together.iq[s])


def oracle_training_gradient(rec, params, freqs, rhs, rx, target, steps, channel_weight):
    """Float64 autograd of the training objective on the oracle: mean over
    systems of log residual + channel_weight * log receiver error."""
    spec = spec_of(rec)
    planes = H.material(spec, rec.c, rec.rho, rec.alpha)
    p = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    rx = torch.as_tensor(rx)
    total = 0.0
    for s in range(len(freqs)):
        op = L.Stencil(H.operator_planes(spec, *planes, freqs[s]), rec.nz, rec.nx, rec.h)
        lp = L.Learned(p, rec.c.astype(np.float64), rec.rho.astype(np.float64), rec.alpha.astype(np.float64),
                       freqs[s], rec.h, rec.c0)
        b = torch.as_tensor(rhs[s].astype(np.complex128))
        res = L.mr_loss(op, lp.apply, b, steps)
        both = L.mr_loss(op, lp.apply, b, steps, rx=rx, target=torch.as_tensor(target[s]))
        total = total + (res + channel_weight * (both - res)) / len(freqs)
    total.backward()
    return float(total.detach()), p.grad.numpy()


# Gradient tolerances against float64 autograd of the oracle (whole vector,
# each parameter block): the FP32 network, and the BF16 network (weights and
# activations rounded to bfloat16, 8 mantissa bits, FP32 accumulation).
GRAD_TOL = {"fp32": (5e-3, 2e-2), "bf16": (3e-2, 1e-1)}


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_training_gradient_matches_oracle_autograd(cuda, gold, precision):
    """All 3,645 parameter gradients of the training loss (three minimal-residual
    steps, residual and receiver terms) from the backward kernels vs float64
    autograd of the oracle, for the FP32 and the BF16 network."""
    from nsrno_b200 import Geometry, Medium
    from nsrno_b200.learned import Batch, loss_and_grad, plane_wave_rhs
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=7, nz=64, nx=96, n_pml=8, n_rx=16, rx_pitch=4)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    geo = med.geometry
    freqs = np.array([4.6e6, 7.9e6])
    angles = np.deg2rad([-12.0, 20.0])
    rng = np.random.default_rng(5)
    params = (gold["params"] * 0.6).astype(np.float32)
    params[8] = math.log(0.12)
    n_rx = len(rec.rx_cols)
    target = rng.standard_normal((2, n_rx)) + 1j * rng.standard_normal((2, n_rx))
    target *= 1e-2
    ft = torch.as_tensor(freqs, device=cuda)
    rhs = (plane_wave_rhs(med, ft, torch.as_tensor(angles, device=cuda)) * geo.h ** 2).to(torch.complex64)
    batch = Batch(med, ft, torch.as_tensor(angles, device=cuda), rhs, geo.rx_index(cuda).long(),
                  torch.as_tensor(target, device=cuda))
    p_dev = torch.as_tensor(params, device=cuda)
    loss, grad, _ = loss_and_grad(p_dev, batch, steps=3, channel_weight=0.7, precision=precision)
    total, ref = oracle_training_gradient(rec, params, freqs, rhs.cpu().numpy(), geo.rx_index("cpu").long().numpy(),
                                          target, steps=3, channel_weight=0.7)
    tol_all, tol_block = GRAD_TOL[precision]
    assert abs(loss - total) < (1e-3 if precision == "fp32" else 1e-2) * abs(total) + 1e-4
    g = grad.cpu().numpy().astype(np.float64)
    assert rel(g, ref) < tol_all, rel(g, ref)
    # each parameter block on its own
    for lo, hi in ((0, 8), (8, 9), (9, 729), (729, 745), (745, 3049), (3049, 3065), (3065, 3641), (3641, 3645)):
        assert rel(g[lo:hi], ref[lo:hi]) < tol_block, (lo, hi, rel(g[lo:hi], ref[lo:hi]))


def test_adam_step_matches_torch(cuda):
    from nsrno_b200.learned import Adam
    g = torch.Generator().manual_seed(0)
    p0 = torch.randn(3645, generator=g)
    grads = [torch.randn(3645, generator=g) * s for s in (1.0, 0.01, 5.0)]
    ours = p0.clone().to(cuda)
    opt = Adam(ours, lr=1e-2, clip=2.0)
    ref = p0.clone().requires_grad_(True)
    topt = torch.optim.Adam([ref], lr=1e-2)
    for gr in grads:
        opt.step(gr.to(cuda))
        ref.grad = gr.clone()
        torch.nn.utils.clip_grad_norm_([ref], 2.0)
        topt.step()
    assert torch.allclose(ours.cpu(), ref.detach(), rtol=1e-5, atol=1e-6)


def test_trained_network_reduces_iterations(cuda):
    """The committed weights against the fixed preconditioner on a held-out
    breast-like medium: same tolerance (1e-6), every system converged, fewer
    BiCGSTAB iterations in total."""
    from nsrno_b200 import Geometry, Medium, solve_batched
    from nsrno_b200.learned import LearnedPreconditioner
    from nsrno_b200.media import breast_bins, breast_record
    bins = breast_bins()[[20, 150, 280]]
    rec = breast_record(seed=999, nz=256, nx=384, n_rx=88, rx_pitch=4, bins=bins, n_angles=3)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    fixed = solve_batched(med, f, th, tolerance=1e-6, max_iterations=4000, n_slots=len(f))
    net = LearnedPreconditioner.load(device=cuda)
    st = net.setup(med, rec.frequencies)
    learned = solve_batched(med, f, th, tolerance=1e-6, max_iterations=4000, n_slots=len(f), learned=st)
    assert fixed.reasons() == ["converged"] * len(f) and learned.reasons() == ["converged"] * len(f)
    assert float(learned.residual.max()) < 1e-6
    it_f = int(fixed.iterations.sum())
    it_l = int(learned.iterations.sum())
    assert it_l < 0.8 * it_f, (it_l, it_f)
    # the receiver IQ of both solves agree to the solve tolerance
    assert rel(learned.iq.cpu().numpy(), fixed.iq.cpu().numpy()) < 1e-4


def test_bf16_network_gains_and_solves(cuda):
    """The BF16 network (bfloat16 weights and activations, FP32 accumulation):
    its gains stay within bfloat16 rounding of the FP32 network's, and solves
    through it converge to the same receiver IQ in as few iterations."""
    from nsrno_b200 import Geometry, Medium, solve_batched
    from nsrno_b200.learned import LearnedPreconditioner
    from nsrno_b200.media import breast_bins, breast_record
    bins = breast_bins()[[20, 150, 280]]
    rec = breast_record(seed=998, nz=256, nx=384, n_rx=88, rx_pitch=4, bins=bins, n_angles=3)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    p32 = LearnedPreconditioner.load(device=cuda, precision="fp32")
    p16 = LearnedPreconditioner.load(device=cuda, precision="bf16")
    s32 = p32.setup(med, rec.frequencies)
    s16 = p16.setup(med, rec.frequencies)
    assert rel(s16.gains.cpu().numpy(), s32.gains.cpu().numpy()) < 2e-2
    r32 = solve_batched(med, f, th, tolerance=1e-6, max_iterations=4000, n_slots=len(f), learned=s32)
    r16 = solve_batched(med, f, th, tolerance=1e-6, max_iterations=4000, n_slots=len(f), learned=s16)
    assert r16.reasons() == ["converged"] * len(f)
    assert int(r16.iterations.sum()) < 1.05 * int(r32.iterations.sum())
    assert rel(r16.iq.cpu().numpy(), r32.iq.cpu().numpy()) < 1e-4
