"""Search logic of the launch-shape autotuner (CPU, a synthetic cost)."""
import json

import pytest

from nsrno_b200 import tune


def fake_cost(cfg):
    """A separable cost with a known minimum; the 512-wide strips of 16 rows
    are 'rejected' by the solver, as an over-large shape would be."""
    if cfg["stencil_width"] == 512 and cfg["stencil_rows"] == 16:
        return None
    c = 1.0
    c += {4: 0.3, 5: 0.2, 6: 0.0}[cfg["stencil_depth"]] if cfg["stencil_width"] == 256 else 0.2
    c += {8: 0.05, 16: 0.0, 32: 0.02, 64: 0.03}[cfg["stencil_rows"]]
    c += 0.01 * cfg["stencil_ctas"]
    c += {0: 0.04, 8: 0.0, 16: 0.04}[cfg["cols_width"]]
    c += {0: 0.0, 1: 0.01}[cfg["cols_staged"]]
    c += {0: 0.0, 1: 0.02}[cfg["rows_staged"]]
    c += {0: 0.03, 2: 0.05, 4: 0.0, 8: 0.02}[cfg["row_tile"]]
    c += {0: 0.0, 1: 0.07, 2: 0.0, 3: 0.01, 4: 0.02}[cfg["slot_groups"]]
    c += {8: 0.02, 16: 0.01, 32: 0.0}[cfg["graph_iterations"]]
    return c


def test_coordinate_descent_finds_the_separable_minimum():
    best, cost, trials = tune.search(fake_cost)
    assert best["stencil_width"] == 256 and best["stencil_depth"] == 6 and best["stencil_rows"] == 16
    assert best["stencil_cols"] in (1, 2)
    assert best["stencil_ctas"] == 0 and best["cols_width"] == 8 and best["row_tile"] == 4
    assert best["graph_iterations"] == 32
    assert cost == pytest.approx(fake_cost(best))
    assert trials[0][0] == tune.DEFAULT
    # every trial is the current best with one parameter group changed; rejected shapes carry no cost
    assert any(c is None for _, c in trials)
    assert all(c is None or c >= cost for _, c in trials)


def test_rejected_default_is_an_error():
    with pytest.raises(RuntimeError):
        tune.search(lambda cfg: None)


def test_split_drops_zero_fields():
    tiles, k = tune.split({**tune.DEFAULT, "cols_width": 8, "graph_iterations": 32})
    assert tiles == {"stencil_width": 256, "stencil_depth": 4, "stencil_cols": 2, "stencil_rows": 64,
                     "cols_width": 8}
    assert k == 32


def test_cache_round_trip(tmp_path, monkeypatch):
    """tuned_config reads a cached entry instead of measuring again."""
    path = tmp_path / "tiles.json"
    key = tune.cache_key("NVIDIA B200", 768, 1024, True, 22)
    path.write_text(json.dumps({key: {"config": {**tune.DEFAULT, "row_tile": 8}, "cost_s": 1.0,
                                      "default_cost_s": 1.2, "gain": 1.2}}))

    class G:
        nz, nx = 768, 1024

    class M:
        geometry = G()
        device = "cuda:0"

    import torch
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "NVIDIA B200")
    monkeypatch.setattr(tune, "tune", lambda *a, **k: pytest.fail("measured despite a cached entry"))
    rec = tune.tuned_config(M(), [1e6], [0.0], learned=object(), n_slots=22, path=path)
    assert rec["cached"] and rec["config"]["row_tile"] == 8 and rec["gain"] == 1.2
