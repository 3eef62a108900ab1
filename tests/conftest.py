"""Shared fixtures.  ``-m gpu`` tests need a CUDA device; the rest run on CPU."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN / "reference_5pt.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from nsrno_b200 import build
    build.build()
    return torch.device("cuda:0")


def spec_of(rec):
    """Oracle spec for a media.Record or solver.Geometry."""
    from oracle import helmholtz_ref as H
    return H.Spec(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, c0=rec.c0, rho0=rec.rho0,
                  pml_strength=rec.pml_strength, face=rec.face, rx_cols=np.asarray(rec.rx_cols),
                  aperture_half_width=rec.aperture_half_width, alpha_power=rec.alpha_power)


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
