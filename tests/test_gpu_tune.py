"""The autotuner on the GPU: it measures, caches, and its choice solves the
same systems as the built-in shapes."""
import numpy as np
import pytest
import torch

from conftest import rel

pytestmark = pytest.mark.gpu


def test_tuned_shapes_solve_the_same_systems(cuda, tmp_path):
    from nsrno_b200 import Geometry, Medium, solve_batched, tune
    from nsrno_b200.media import breast_record
    rec = breast_record(seed=21, nz=256, nx=384, n_pml=16, n_rx=48, rx_pitch=4, n_angles=3)
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=cuda)
    f, th = rec.systems()
    f, th = f[::97][:6], th[::97][:6]
    groups = [("stencil", [dict(stencil_width=512, stencil_depth=4, stencil_cols=2, stencil_rows=8),
                           dict(stencil_width=256, stencil_depth=6, stencil_cols=1, stencil_rows=32)]),
              ("row_tile", [dict(row_tile=2)]), ("graph_iterations", [dict(graph_iterations=8)])]
    path = tmp_path / "tiles.json"
    first = tune.tuned_config(med, f, th, n_slots=6, path=path, iterations=12, repeats=1, groups=groups)
    assert not first["cached"] and len(first["trials"]) == 5 and first["cost_s"] > 0
    assert first["gain"] >= 1.0
    again = tune.tuned_config(med, f, th, n_slots=6, path=path)
    assert again["cached"] and again["config"] == first["config"]
    tiles, k = tune.split(first["config"])
    base = solve_batched(med, f, th, tolerance=1e-7, n_slots=6, max_iterations=4000)
    got = solve_batched(med, f, th, tolerance=1e-7, n_slots=6, max_iterations=4000, tiles=tiles,
                        graph_iterations=k)
    assert got.reasons() == ["converged"] * len(f)
    assert rel(got.iq.cpu().numpy(), base.iq.cpu().numpy()) < 1e-5
