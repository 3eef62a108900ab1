"""Generate golden vectors of the learned preconditioner from the reference
implementation (run on a machine that has the reference checked out; the
tests only read the vectors it writes).

    python tests/golden/make_golden_learned.py REFERENCE_CHECKOUT

Writes ``tests/golden/reference_learned.npz``.  The reference's own
``LearnedPreconditioner`` (nsrno/conditioned_wave.py:94-117) and ``learned_apply``
(nsrno/dense_wave.py:150-165), in float64 with seeded non-zero parameters, are
evaluated on a system whose geometry carries the 5-point symbols
(``lap = -4 (sin^2(qx/2) + sin^2(qz/2))/h^2``, ``|Dx|^2 = 4 sin^2(qx/2)/h^2``) and
a mask of ones:

* ``params``            -- the flat parameter vector in state_dict order;
* ``c, rho, alpha, frequency, h, c0`` -- the medium and grid;
* ``maps``              -- ``network.context(avg_pool2d(context, 8))`` [4, h/8, w/8];
* ``probe``, ``apply``  -- a seeded complex field and ``setup(system)(probe)``;
* ``adjoint``           -- ``learned_apply(network, system, adjoint=True)(probe)``.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import torch
from torch.nn import functional as F


def main(reference_root):
    sys.path.insert(0, str(reference_root))
    from nsrno.conditioned_wave import LearnedPreconditioner
    from nsrno.dense_wave import learned_apply
    from nsrno.wave_operator import C0, RHO0

    torch.manual_seed(11)
    net = LearnedPreconditioner().double()
    with torch.no_grad():
        for name, p in net.named_parameters():
            if name == "log_shift":
                p.fill_(math.log(0.21))
            elif name == "spectral":
                p.copy_(0.4 * torch.randn_like(p))
            else:
                p.copy_(0.35 * torch.randn_like(p))
    H, W, h, c0, f = 48, 64, 5e-5, 1500.0, 5.3e6
    rng = np.random.default_rng(4)
    zz, xx = np.meshgrid(np.arange(H), np.arange(W), indexing="ij")
    c = 1500 + 60 * np.sin(zz / 7.0) * np.cos(xx / 9.0) + 10 * rng.standard_normal((H, W))
    rho = 1000 + 50 * np.cos(zz / 5.0 + xx / 11.0) + 5 * rng.standard_normal((H, W))
    alpha = 0.5 + 0.3 * rng.random((H, W))
    qx = 2 * math.pi * torch.fft.fftfreq(W, dtype=torch.float64)
    qz = 2 * math.pi * torch.fft.fftfreq(H, dtype=torch.float64)
    dx = (2j * torch.sin(qx / 2) * torch.exp(0.5j * qx) / h)[None, :]
    lap = -((4 * torch.sin(qx / 2) ** 2 / h ** 2)[None, :] + (4 * torch.sin(qz / 2) ** 2 / h ** 2)[:, None])
    g = SimpleNamespace(H=H, W=W, lap=lap, Dx=dx, mask=torch.ones(H, W, dtype=torch.float64))
    k0 = 2 * math.pi * f / c0
    tc, tr, ta = (torch.tensor(v, dtype=torch.float64) for v in (c, rho, alpha))
    system = SimpleNamespace(c=tc, rho=tr, alpha=ta, frequency=f, g=g, k0=k0)
    probe = torch.tensor(rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W)))
    with torch.no_grad():
        apply = net.setup(system)(probe)
        ctx = torch.stack(((tc / C0).log() / .06, (tr / RHO0).log() / .08, torch.log1p(ta),
                           torch.ones_like(tc) * (f / 6e6 - 1), g.mask))[None]
        maps = net.context(F.avg_pool2d(ctx, 8))[0]
        # learned_apply converts the medium to float32 and runs the network in
        # the dtype of its weights; a float32 copy of the network is used there.
        net32 = LearnedPreconditioner()
        net32.load_state_dict({k: v.float() for k, v in net.state_dict().items()})
        g32 = SimpleNamespace(H=H, W=W, lap=lap.float(), Dx=dx.to(torch.complex64), mask=g.mask.float())
        s32 = SimpleNamespace(c=tc, rho=tr, alpha=ta, frequency=f, g=g32, k0=k0)
        adjoint = learned_apply(net32, s32, adjoint=True)(probe.to(torch.complex64))
        forward32 = learned_apply(net32, s32)(probe.to(torch.complex64))
    params = torch.cat([v.reshape(-1) for v in net.state_dict().values()])
    out = dict(params=params.numpy(), c=c, rho=rho, alpha=alpha, frequency=f, h=h, c0=c0,
               maps=maps.numpy(), probe=probe.numpy(), apply=apply.numpy(),
               adjoint=adjoint.numpy().astype(np.complex128), forward32=forward32.numpy().astype(np.complex128))
    path = Path(__file__).resolve().parent / "reference_learned.npz"
    np.savez_compressed(path, **out)
    print(path, {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT")
    main(sys.argv[1])
