"""The learned-preconditioner oracle pinned against the reference's own module."""
import math

import numpy as np
import pytest
import torch
from torch.nn import functional as F

from conftest import GOLDEN, rel
from oracle import learned_ref as L


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN / "reference_learned.npz") as z:
        return {k: z[k] for k in z.files}


def learned_of(gold, params=None):
    p = torch.as_tensor(gold["params"] if params is None else params, dtype=torch.float64)
    return L.Learned(p, gold["c"], gold["rho"], gold["alpha"], float(gold["frequency"]), float(gold["h"]),
                     float(gold["c0"]))


def kh2_of(gold):
    return (2 * math.pi * float(gold["frequency"]) / float(gold["c0"]) * float(gold["h"])) ** 2


def test_parameter_count_matches_reference():
    assert L.N_PARAMS == 3645


def test_network_maps_match_reference(gold):
    lp = learned_of(gold)
    assert rel(lp.maps.numpy(), gold["maps"]) < 1e-13


def test_apply_is_the_conjugate_map_of_the_reference(gold):
    lp = learned_of(gold)
    probe = torch.as_tensor(gold["probe"])
    ours = lp.apply(probe.conj()).numpy()
    assert rel(ours, np.conj(gold["apply"]) / kh2_of(gold)) < 1e-12
    # learned_apply (float32 in the reference) is the same operator
    assert rel(ours, np.conj(gold["forward32"]) / kh2_of(gold)) < 2e-5


def test_adjoint_matches_reference_learned_apply(gold):
    lp = learned_of(gold)
    probe = torch.as_tensor(gold["probe"])
    ours = lp.adjoint(probe.conj()).numpy()
    assert rel(ours, np.conj(gold["adjoint"]) / kh2_of(gold)) < 2e-5


def test_adjoint_identity(gold):
    lp = learned_of(gold)
    g = torch.Generator().manual_seed(1)
    p = torch.randn(48, 64, generator=g, dtype=torch.float64) + 1j * torch.randn(48, 64, generator=g, dtype=torch.float64)
    q = torch.randn(48, 64, generator=g, dtype=torch.float64) + 1j * torch.randn(48, 64, generator=g, dtype=torch.float64)
    left = torch.vdot(q.reshape(-1), lp.apply(p).reshape(-1))
    right = torch.vdot(lp.adjoint(q).reshape(-1), p.reshape(-1))
    assert abs(left - right) < 1e-12 * abs(left)


def test_building_blocks_equal_torch_functional():
    g = torch.Generator().manual_seed(2)
    x = torch.randn(5, 7, 9, generator=g, dtype=torch.float64)
    w = torch.randn(16, 5, 3, 3, generator=g, dtype=torch.float64)
    b = torch.randn(16, generator=g, dtype=torch.float64)
    assert torch.allclose(L.conv3x3(x, w, b), F.conv2d(x[None], w, b, padding=1)[0], atol=1e-12)
    m = torch.randn(4, 6, 8, generator=g, dtype=torch.float64)
    for size in ((48, 64), (50, 61), (768, 1024)):
        ref = F.interpolate(m[None], size=size, mode="bilinear", align_corners=False)[0]
        assert torch.allclose(L.upsample(m, *size), ref, atol=1e-12)
    ctx = torch.randn(5, 52, 67, generator=g, dtype=torch.float64)
    assert torch.allclose(L.pool8(ctx), F.avg_pool2d(ctx[None], 8)[0], atol=1e-12)


def test_untrained_network_is_the_fixed_preconditioner(gold):
    """Zero last layer, zero spectral weights and log(0.15): the fixed shifted-Laplace inverse."""
    lp = learned_of(gold, L.initial_parameters().numpy())
    nz, nx = gold["c"].shape
    h, f, c0 = float(gold["h"]), float(gold["frequency"]), float(gold["c0"])
    k0 = 2 * math.pi * f / c0
    qx = 2 * math.pi * np.fft.fftfreq(nx)
    qz = 2 * math.pi * np.fft.fftfreq(nz)
    sym = -4 * (np.sin(qz / 2)[:, None] ** 2 + np.sin(qx / 2)[None, :] ** 2) + (k0 * h) ** 2 * (1 + 0.15j)
    probe = gold["probe"]
    fixed = np.fft.ifft2(np.fft.fft2(probe) / sym)
    assert rel(lp.apply(torch.as_tensor(probe)).numpy(), fixed) < 1e-13
