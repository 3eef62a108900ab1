"""Generate golden vectors of the reference's 8th-order dense operator
(run in a container that has the reference checked out; not needed where the tests only run).

    python tests/golden/make_golden_dense.py REFERENCE_CHECKOUT

Writes ``tests/golden/reference_dense.npz`` with a synthetic acquisition spec
(the V5 metadata is not part of the reference checkout), a seeded medium and
attenuation map, and, for a seeded complex128 probe field p on the padded
grid, ``projected_operator(system, p)`` and ``adjoint_operator(system, p)``
(nsrno/dense_wave.py:66-82, nsrno/conditioned_wave.py:52-80) restricted to the
native (masked) region -- outside it both operators are the identity.
The probe is ``default_rng(PROBE_SEED)`` normal real + 1j normal imag, [H, W].
Also stored, at the first frequency: the fixed preconditioner of the probe,
the acquisition right-hand side ``S(line) - S0(line) - A p_ref + A0 p_ref`` of
seeded lines and masked reference fields, the source term alone, a GMRES
solve converged to 1e-10, and the implicit gradient of ImplicitChannels'
backward for seeded forward and adjoint fields (the same lines and reference
fields).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

PROBE_SEED = 20261203
ASSEMBLY_SEED = 77
GRADIENT_SEED = 4242
SPEC = {"medium_shape": [32, 40], "dx_m": 5e-5, "x0_m": -0.001, "z0_m": -0.0002, "native_dt_s": 2.5e-9,
        "pml": 6, "eta_per_unit_alpha": [0.012, 0.021], "taus_s": [2.0e-8, 1.5e-7],
        "source_c_lookup_zx": [10, 20]}
FREQS = [4.5e6, 7.2e6]


def main(reference_root):
    sys.path.insert(0, str(reference_root))
    import torch
    from nsrno.conditioned_wave import ConditionedFrequencySystem, FrequencyGeometry
    from nsrno.dense_wave import adjoint_operator, projected_operator

    torch.set_default_dtype(torch.float64)
    g = FrequencyGeometry(SPEC)
    h, w = SPEC["medium_shape"]
    rng = np.random.default_rng(5)
    c = 1540.0 + 60.0 * rng.standard_normal((h, w))
    rho = 1000.0 + 50.0 * rng.standard_normal((h, w))
    alpha = rng.uniform(0.2, 1.2, (h, w))
    medium = torch.tensor(np.stack((c, rho)))
    out = {"spec": json.dumps(SPEC), "medium": np.stack((c, rho)), "alpha": alpha, "freqs": np.array(FREQS),
           "probe_seed": PROBE_SEED, "H": g.H, "W": g.W, "pz": g.pz, "px": g.px}
    prng = np.random.default_rng(PROBE_SEED)
    p = prng.standard_normal((g.H, g.W)) + 1j * prng.standard_normal((g.H, g.W))
    pt = torch.tensor(p)[None]
    for k, f in enumerate(FREQS):
        s = ConditionedFrequencySystem(g, medium, torch.tensor(alpha), f)
        y = projected_operator(s, pt)[0].numpy()
        yh = adjoint_operator(s, pt)[0].numpy()
        inner = (slice(g.pz, g.pz + h), slice(g.px, g.px + w))
        out[f"y{k}"] = y[inner]
        out[f"yh{k}"] = yh[inner]
        # outside the native region both operators leave p unchanged
        mask = np.zeros((g.H, g.W), bool)
        mask[inner] = True
        assert np.allclose(y[~mask], p[~mask]) and np.allclose(yh[~mask], p[~mask])
    # Fixed preconditioner, acquisition assembly and a converged GMRES solve
    # (nsrno/conditioned_wave.py:82-92, nsrno/dense_wave.py:46-62,
    # nsrno/wave_solver.py:9-36) at the first frequency, complex128.
    from nsrno.dense_wave import source_rhs
    from nsrno.wave_solver import gmres
    s = ConditionedFrequencySystem(g, medium, torch.tensor(alpha), FREQS[0])
    out["precondition"] = s.fixed_preconditioner()(pt)[0].numpy()
    uniform = torch.empty_like(medium)
    uniform[0] = 1540.0
    uniform[1] = 1000.0
    s0 = ConditionedFrequencySystem(g, uniform, torch.full_like(torch.tensor(alpha), 0.002), FREQS[0])
    arng = np.random.default_rng(ASSEMBLY_SEED)
    line = torch.tensor(arng.standard_normal((2, w)) + 1j * arng.standard_normal((2, w)))
    pref = torch.tensor(arng.standard_normal((2, g.H, g.W)) + 1j * arng.standard_normal((2, g.H, g.W)))
    pref = pref * g.mask
    rhs = source_rhs(s, line) - source_rhs(s0, line) - projected_operator(s, pref) + projected_operator(s0, pref)
    out.update(assembly_line=line.numpy(), assembly_pref=pref.numpy(), assembly_rhs=rhs.numpy(),
               source=source_rhs(s, line).numpy())
    trace = []
    b = rhs[:1]
    x, reason = gmres(lambda v: projected_operator(s, v), s.fixed_preconditioner(), b, torch.zeros_like(b),
                      lambda n, u, r: trace.append(r), restart=32, max_cycles=200, tolerance=1e-10)
    assert reason == "converged", trace[-1]
    out["solve_rhs"] = b.numpy()
    out["solve_x"] = x.numpy()
    # The implicit gradient of ImplicitChannels.backward (nsrno/dense_wave.py:250-255)
    # for seeded fields: d/d(medium) of -Re sum conj(lam) mask (A(m)(mask (u + pref)) - S(m) line).
    grng = np.random.default_rng(GRADIENT_SEED)
    shape = (2, g.H, g.W)
    u = torch.tensor(grng.standard_normal(shape) + 1j * grng.standard_normal(shape))
    lam = torch.tensor(grng.standard_normal(shape) + 1j * grng.standard_normal(shape))
    material = medium.clone().requires_grad_(True)
    physical = ConditionedFrequencySystem(g, material, torch.tensor(alpha), FREQS[0])
    residual = physical(g.mask * (u + pref)) - source_rhs(physical, line)
    scalar = -(lam.conj() * g.mask * residual).real.sum()
    out.update(grad_u=u.numpy(), grad_lam=lam.numpy(),
               grad_medium=torch.autograd.grad(scalar, material)[0].numpy())
    path = Path(__file__).resolve().parent / "reference_dense.npz"
    np.savez_compressed(path, **out)
    print(path, {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT")
    main(sys.argv[1])
