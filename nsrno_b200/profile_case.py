"""A small, fixed workload of the batched solver for kernel profilers.

``python -m nsrno_b200.profile_case [--learned] [--systems 22] [--iterations 12]``
solves ``--systems`` (frequency, angle) systems of the 1024 (x) x 768 (z)
breast record, spread over its band, for exactly ``--iterations`` BiCGSTAB
iterations (an unreachable tolerance) with the host-polled loop, in which
every kernel is a separate launch that a profiler can capture (kernels inside
the conditional graph of the default device-side loop cannot be captured one
by one).  With 22 systems the slots and slot groups are those of the
benchmark's steady state, so a capture such as
``ncu -k regex:k_stn -s 6 -c 2 python -m nsrno_b200.profile_case`` sees the
benchmark's launches on a workload of a few GB.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def run(learned=False, systems=22, iterations=12, graph_iterations=4, precision=None, tiles=None, device=None):
    import torch
    from . import Geometry, Medium, solve_batched
    from .media import breast_record
    device = torch.device(device or "cuda:0")
    rec = breast_record()
    med = Medium(Geometry.from_record(rec), rec.c, rec.rho, rec.alpha, device=device)
    f, a = rec.systems()
    pick = np.linspace(0, len(f) - 1, systems).round().astype(int)
    f, a = f[pick], a[pick]
    setup = None
    if learned:
        from .learned import LearnedPreconditioner
        setup = LearnedPreconditioner.load(device=device, precision=precision).setup(med, np.unique(f))
    r = solve_batched(med, f, a, tolerance=1e-30, max_iterations=iterations, n_slots=systems,
                      graph_iterations=graph_iterations, learned=setup, tiles=tiles, blocking=True)
    torch.cuda.synchronize()
    return {"systems": systems, "iterations": iterations, "learned": bool(learned),
            "reasons": sorted(set(r.reasons())), "loop_ms": r.extra["stats"]["loop_ms"]}


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--learned", action="store_true", help="learned preconditioner (committed weights)")
    ap.add_argument("--precision", choices=["fp32", "bf16"], default=None)
    ap.add_argument("--systems", type=int, default=22)
    ap.add_argument("--iterations", type=int, default=12)
    ap.add_argument("--tiles", type=str, default=None, help="launch shapes as JSON (NsrTiles fields)")
    a = ap.parse_args()
    tiles = json.loads(a.tiles) if a.tiles else None
    print(json.dumps(run(a.learned, a.systems, a.iterations, precision=a.precision, tiles=tiles)))


if __name__ == "__main__":
    main()
