"""Autotuner of the batched solver's launch shapes.

The batched BiCGSTAB (``nsr_solve_batched``) runs nine launches per
iteration whose shapes are free parameters (:class:`nsrno_b200._lib.NsrTiles`):
the stencil's work item (columns ``stencil_width``, rows ``stencil_rows``),
its copy-ring depth ``stencil_depth`` and resident CTAs per SM, the
column-transform tile ``cols_width``, the row-transform tile ``row_tile``,
whether the column and row transforms run their end stages between registers
and global memory (``cols_staged``, ``rows_staged``), the
number of slot groups on graph branches, plus the CUDA-graph length
``graph_iterations``.  The best choice depends on the grid, the GPU and the
preconditioner, so it is measured: :func:`tune` times a fixed number of
iterations of a full set of resident systems for each candidate (device
events around the graph-launched loop) and keeps the fastest, searching one
parameter group at a time from the built-in defaults (coordinate descent).
:func:`tuned_config` caches the choice per (GPU, grid, preconditioner) in a
JSON file.

Shapes of the transforms and of the slot groups leave every system's
arithmetic unchanged; stencil shapes regroup the FP64 partial sums of the
inner products, so results agree to rounding of those sums.

The reference has no counterpart: its solver fixes ``restart=24/32`` and its
FFT paddings (nsrno/dense_wave.py:19,216).
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

# Parameter groups searched in this order; each candidate is a partial NsrTiles
# dict (plus graph_iterations) merged into the current best.
STENCIL_SHAPES = ([dict(stencil_width=w, stencil_depth=d, stencil_cols=2, stencil_rows=r)
                   for (w, d) in ((256, 4), (256, 5), (256, 6), (512, 4))
                   for r in (16, 32, 64)] +
                  [dict(stencil_width=256, stencil_depth=4, stencil_cols=1, stencil_rows=32)])
GROUPS = [
    ("stencil", STENCIL_SHAPES),
    ("stencil_ctas", [dict(stencil_ctas=0), dict(stencil_ctas=1), dict(stencil_ctas=2)]),
    ("cols_width", [dict(cols_width=8), dict(cols_width=16)]),
    ("cols_staged", [dict(cols_staged=1), dict(cols_staged=0)]),
    ("rows_staged", [dict(rows_staged=1), dict(rows_staged=0)]),
    ("row_tile", [dict(row_tile=r) for r in (2, 4, 8)]),
    ("slot_groups", [dict(slot_groups=g) for g in (1, 2, 3, 4)]),
    ("graph_iterations", [dict(graph_iterations=k) for k in (8, 16, 32)]),
]
DEFAULT = dict(stencil_width=256, stencil_depth=4, stencil_cols=2, stencil_rows=64, stencil_ctas=0, cols_width=0,
               cols_staged=0, rows_staged=0, row_tile=0, slot_groups=0, graph_iterations=16)
TILE_KEYS = ("stencil_width", "stencil_depth", "stencil_cols", "stencil_rows", "stencil_ctas", "cols_width",
             "cols_staged", "rows_staged", "row_tile", "slot_groups")


def search(measure, groups=GROUPS, start=None, repeats=1):
    """Coordinate descent: for each parameter group in turn, time every candidate
    merged into the current best and keep the fastest.  ``measure(config)``
    returns a cost (lower is better) or ``None`` when the configuration is
    rejected.  Returns ``(best_config, best_cost, trials)`` with ``trials`` a
    list of ``(config, cost)``."""
    best = dict(DEFAULT if start is None else start)
    trials = []

    def cost_of(cfg):
        costs = [measure(dict(cfg)) for _ in range(max(1, repeats))]
        costs = [c for c in costs if c is not None]
        cost = min(costs) if costs else None
        trials.append((dict(cfg), cost))
        return cost

    best_cost = cost_of(best)
    if best_cost is None:
        raise RuntimeError("the default launch shapes were rejected")
    for _, candidates in groups:
        for cand in candidates:
            cfg = {**best, **cand}
            if cfg == best:
                continue
            cost = cost_of(cfg)
            if cost is not None and cost < best_cost:
                best, best_cost = cfg, cost
    return best, best_cost, trials


def split(config):
    """(tiles dict for solve_batched, graph_iterations) of a tuned configuration."""
    tiles = {k: int(config[k]) for k in TILE_KEYS if int(config.get(k, 0))}
    return tiles, int(config.get("graph_iterations", 16))


def measure_iteration(medium, freqs, angles, config, learned=None, n_slots=22, iterations=24, shift=None):
    """Device seconds per system-iteration of ``config``: ``n_slots`` systems,
    every one running exactly ``iterations`` BiCGSTAB iterations (an
    unreachable tolerance), timed by events around the graph-launched loop.
    Returns ``None`` if the solver rejects the shapes."""
    import torch
    from .solver import DEFAULT_SHIFT, solve_batched
    freqs = np.resize(np.asarray(freqs, dtype=np.float64), n_slots)
    angles = np.resize(np.asarray(angles, dtype=np.float64), n_slots)
    tiles, graph_iterations = split(config)
    try:
        r = solve_batched(medium, freqs, angles, tolerance=1e-30, max_iterations=iterations, n_slots=n_slots,
                          graph_iterations=graph_iterations, learned=learned, tiles=tiles,
                          shift=DEFAULT_SHIFT if shift is None else shift, blocking=True)
    except (RuntimeError, ValueError):
        return None
    torch.cuda.synchronize()
    return r.extra["stats"]["loop_ms"] * 1e-3 / (iterations * n_slots)


def cache_path():
    env = os.environ.get("NSRNO_B200_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "nsrno_b200" / "tiles.json"


def cache_key(device_name, nz, nx, learned, n_slots):
    return f"{device_name}|{nz}x{nx}|{'learned' if learned else 'fixed'}|slots{n_slots}"


def tune(medium, freqs, angles, learned=None, n_slots=22, iterations=24, repeats=2, groups=GROUPS):
    """Measure the candidates on ``medium`` (systems drawn from ``freqs``,
    ``angles``) and return a record with the best configuration, its cost and
    the default's cost (seconds per system-iteration) and every trial."""
    # one untimed solve loads the module and warms the allocator
    measure_iteration(medium, freqs, angles, DEFAULT, learned, n_slots, iterations=4)
    started = time.perf_counter()
    best, best_cost, trials = search(
        lambda cfg: measure_iteration(medium, freqs, angles, cfg, learned, n_slots, iterations),
        groups=groups, repeats=repeats)
    default_cost = next(c for cfg, c in trials if cfg == {**DEFAULT})
    return {"config": best, "cost_s": best_cost, "default_cost_s": default_cost, "gain": default_cost / best_cost,
            "trials": [{"config": c, "cost_s": v} for c, v in trials],
            "seconds": time.perf_counter() - started}


def tuned_config(medium, freqs, angles, learned=None, n_slots=22, refresh=False, path=None, **kw):
    """The cached tuned configuration of this GPU, grid and preconditioner
    (tuning on a miss, or when ``refresh``)."""
    import torch
    path = Path(path) if path is not None else cache_path()
    g = medium.geometry
    key = cache_key(torch.cuda.get_device_name(medium.device), g.nz, g.nx, learned is not None, n_slots)
    table = {}
    if path.exists():
        try:
            table = json.loads(path.read_text())
        except (OSError, ValueError):
            table = {}
    if not refresh and key in table:
        return {**table[key], "cached": True}
    record = tune(medium, freqs, angles, learned=learned, n_slots=n_slots, **kw)
    entry = {k: record[k] for k in ("config", "cost_s", "default_cost_s", "gain")}
    table[key] = entry
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home still gets the tuned shapes for this process
    return {**entry, "cached": False, "trials": record["trials"], "seconds": record["seconds"]}
