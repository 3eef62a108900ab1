"""Throughput of the batched frequency-domain Helmholtz solve on B200.

Workload: the synthetic breast record, 1024 (x) x 768 (z) nodes at 0.05 mm,
11 plane-wave angles x 294 frequency bins (4.015-8.896 MHz) = 3234 systems,
BiCGSTAB to a true relative residual of 1e-6.  One step solves a batch of
SYSTEMS_PER_STEP systems (4 bins x 11 angles, bins spread over the band by a
fixed stride permutation) through the resident-slot queue.  Under torchrun
every rank takes different bins (weak scaling, no collective on the data path).

Two arms run on the same GPU and the same steps: the headline "learned-init"
arm (the trained learned preconditioner: its network set-up for the step's
bins is inside the timed region) and the "plain Krylov" arm (the fixed
shifted-Laplace preconditioner, shift 0.15), reported under ``plain_krylov``.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "converged Helmholtz solves/s at rel-res 1e-6: learned-init vs plain Krylov"
UNIT = "solves/s"
TOL = 1e-6
BINS_PER_STEP = 4
N_ANGLES = 11
SYSTEMS_PER_STEP = BINS_PER_STEP * N_ANGLES
N_SLOTS = 22
MAX_ITERS = 4000
PROFILE_ITERS = 10
FALLBACK_HBM_GBS = 6650.0
# Algorithmic bytes per node of one BiCGSTAB iteration and per kernel launch,
# per resident system (complex64 vectors; coefficient planes counted once per
# launch and listed separately): fwd h0 reads r,v,t,p,y and writes r,p,y,w;
# cols and rinv read and write w; inv h0 reads z (= w after rinv), rhat and
# writes v; fwd h1 reads r,v and writes w; inv h1 reads z, rhat, r, v and
# writes t.  res h1 (the FP64 true residual) has no work in the timed
# iterations of a fresh batch.
KERNEL_BYTES = {"fwd_h0": 72, "cols_h0": 16, "rinv_h0": 16, "inv_h0": 24, "fwd_h1": 24, "cols_h1": 16,
                "rinv_h1": 16, "res_h1": 0, "inv_h1": 40}
# The learned preconditioner adds one complex64 read per node to every fwd
# launch (inner gain), every cols launch (the multiplier plane of the slot's
# system) and every rinv launch (outer gain).
LEARNED_BYTES = {k: v + (8 if k.startswith(("fwd", "cols", "rinv")) else 0) for k, v in KERNEL_BYTES.items()}
COEF_BYTES = {"inv_h0": 12, "inv_h1": 12}
LEARNED_SETUP_LAUNCHES = 5     # pool, three convolutions, gains


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cpu-sample-bins", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain-Krylov comparison arm")
    p.add_argument("--plain-only", action="store_true",
                   help="run only the plain-Krylov arm (for profiling it); prints a short line, not the bench line")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def bin_permutation(n_bins=294, stride=151):
    """Fixed stride permutation so that consecutive steps sample the whole band."""
    return (np.arange(n_bins) * stride) % n_bins


def step_systems(record, step, rank, world):
    """(freqs, angles) of one step on one rank, highest frequency first."""
    perm = bin_permutation(len(record.frequencies))
    first = (step * world + rank) * BINS_PER_STEP
    bins = [perm[(first + k) % len(perm)] for k in range(BINS_PER_STEP)]
    f = np.repeat(record.frequencies[bins], N_ANGLES)
    a = np.tile(record.angles, BINS_PER_STEP)
    order = np.argsort(-f, kind="stable")
    return f[order], a[order]


# ---------------------------------------------------------------------------
# GPU clocks sampled during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def peak_hbm():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(arm, kernel):
    """DRAM bytes per node and resident system of one kernel of one arm, from the committed ncu summaries."""
    pat = r"traffic_bytes_per_node_per_system:\s*([0-9.eE+-]+)\s*kernel:\s*(\w+)\s*arm:\s*(\w+)"
    for path in sorted((ROOT / "profiles").glob("*.md")):
        for m in re.finditer(pat, path.read_text()):
            if m.group(3) == arm and m.group(2) == kernel:
                return float(m.group(1))
    return None


# ---------------------------------------------------------------------------
# CPU arm: the reference algorithm of the path (assemble, one SuperLU factor
# per frequency shared by all angles, solve) restated by the oracle.
# ---------------------------------------------------------------------------
def _cpu_one_bin(args):
    import os as _os
    _os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import helmholtz_ref as H
    from nsrno_b200.media import breast_record
    rec = breast_record()
    spec = H.Spec(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, c0=rec.c0, rho0=rec.rho0,
                  pml_strength=rec.pml_strength, face=rec.face, rx_cols=rec.rx_cols,
                  aperture_half_width=rec.aperture_half_width, alpha_power=rec.alpha_power)
    fields, seconds, res = H.time_lu_frequency(spec, rec.c, rec.rho, rec.alpha, rec.frequencies[args], rec.angles)
    return seconds, res, len(rec.angles)


def cpu_sample(n_bins, processes):
    """Wall time of n_bins frequencies (11 angles each) on `processes` host processes."""
    import multiprocessing as mp
    perm = bin_permutation()
    bins = [int(perm[k]) for k in range(n_bins)]
    t0 = time.perf_counter()
    if processes <= 1:
        out = [_cpu_one_bin(b) for b in bins]
    else:
        with mp.get_context("spawn").Pool(processes) as pool:
            out = pool.map(_cpu_one_bin, bins)
    wall = time.perf_counter() - t0
    solves = sum(o[2] for o in out)
    return solves / wall, wall, solves, max(o[1] for o in out)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    procs = max(1, min(cores, 8, args.cpu_sample_bins * max(1, args.steps)))
    # each step: one bin per process (11 angles each), in parallel
    for _ in range(args.warmup):
        pass  # the factorisation has no warm state worth priming; warm-up steps are skipped
    values = []
    t_total = 0.0
    solves_total = 0
    for _ in range(max(1, args.steps)):
        v, wall, solves, res = cpu_sample(procs, procs)
        values.append(v)
        t_total += wall
        solves_total += solves
    value = solves_total / t_total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "breast 1024x768 dx=0.05mm, 11 angles x 294 bins; CPU: assemble + SuperLU "
                                   "factor per bin + 11 angle solves (theranostic/wave.py:240-273 restated)",
                       "bins_per_step": procs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                             "sample": f"{procs} bins x 11 angles per step on {procs} processes"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from nsrno_b200 import Geometry, Medium, Workspace, _lib, solve_batched
    from nsrno_b200.learned import LearnedPreconditioner
    from nsrno_b200.media import breast_record

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rec = breast_record()
    geo = Geometry.from_record(rec)
    med = Medium(geo, rec.c, rec.rho, rec.alpha, device=dev)
    net = LearnedPreconditioner.load(device=dev)
    ws = Workspace()

    def one_step(step, learned, medium=med, profile=0, host=False):
        f, a = step_systems(rec, step, rank, world)
        if host:
            f = torch.from_numpy(f).pin_memory().to(dev, non_blocking=True)
            a = torch.from_numpy(a).pin_memory().to(dev, non_blocking=True)
        setup = None
        if learned:
            setup = net.setup(medium, torch.unique(torch.as_tensor(f, device=dev)))
        return solve_batched(medium, f, a, tolerance=TOL, max_iterations=MAX_ITERS, n_slots=N_SLOTS,
                             profile_iterations=profile, workspace=ws, learned=setup)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    stream = torch.cuda.current_stream()

    def timed(learned, sample_clocks=False):
        for w in range(args.warmup):
            one_step(-(w + 1), learned)
        barrier()
        clocks = ClockSampler(local) if sample_clocks else None
        if clocks:
            clocks.start()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        results = []
        t0.record(stream)
        for k in range(args.steps):
            results.append(one_step(k, learned, profile=PROFILE_ITERS))
        t1.record(stream)
        barrier()
        clock_info = clocks.stop() if clocks else None
        ms_t = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        return float(ms_t), results, clock_info

    n = rec.nz * rec.nx
    slots = min(N_SLOTS, SYSTEMS_PER_STEP)
    peak, peak_kind = peak_hbm()
    solves = SYSTEMS_PER_STEP * args.steps * world

    def summarise(ms_max, results, per_node):
        status = torch.cat([r.status for r in results]).cpu().numpy()
        iters = torch.cat([r.iterations for r in results]).cpu().numpy()
        resid = torch.cat([r.residual for r in results]).cpu().numpy()
        # per-kernel durations measured by events between launches (first iterations of every step)
        kms = {k: float(np.mean([r.extra["stats"]["kernel_ms"][k] for r in results])) for k in per_node}
        alg = {k: n * (per_node[k] * slots + COEF_BYTES.get(k, 0)) for k in per_node}
        dominant = max(kms, key=kms.get)
        iter_ms = sum(kms.values())
        return dict(value=solves / (ms_max / 1e3), ms_per_step=ms_max / max(1, args.steps), kms=kms, alg=alg,
                    dominant=dominant, achieved=alg[dominant] / (kms[dominant] / 1e3) / 1e9,
                    iteration_achieved=sum(alg.values()) / (iter_ms / 1e3) / 1e9,
                    launches=int(sum(r.extra["stats"]["launches"] for r in results)),
                    solves={"total": int(len(status)), "converged": int((status == _lib.CONVERGED).sum()),
                            "iterations_mean": float(iters.mean()), "iterations_max": int(iters.max()),
                            "residual_max": float(resid.max())})

    if args.plain_only:
        ms_p, res_p, _ = timed(False)
        P = summarise(ms_p, res_p, KERNEL_BYTES)
        if rank == 0:
            print(json.dumps({"arm": "plain", "value": P["value"], "unit": UNIT, "kernel_ms": P["kms"],
                              "solves": P["solves"]}), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    ms_l, res_l, clock_info = timed(True, sample_clocks=True)
    L = summarise(ms_l, res_l, LEARNED_BYTES)
    P = None
    if not args.no_plain:
        ms_p, res_p, _ = timed(False)
        P = summarise(ms_p, res_p, KERNEL_BYTES)
    value = L["value"]
    dominant = L["dominant"]
    achieved = L["achieved"]
    launches = L["launches"] + LEARNED_SETUP_LAUNCHES * args.steps
    traffic_per_node = profiled_traffic("learned", dominant)
    traffic = None if traffic_per_node is None else traffic_per_node * n * slots
    plain_traffic = None
    if P is not None:
        tp = profiled_traffic("plain", P["dominant"])
        plain_traffic = None if tp is None else tp * n * slots

    # end to end through the public API with host buffers (learned arm)
    e2e_value = None
    h2d = d2h = 0
    if args.steps > 0:
        host_c = torch.from_numpy(rec.c).pin_memory()
        host_r = torch.from_numpy(rec.rho).pin_memory()
        host_a = torch.from_numpy(rec.alpha).pin_memory()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.steps):
            m2 = Medium(geo, host_c.to(dev, non_blocking=True), host_r.to(dev, non_blocking=True),
                        host_a.to(dev, non_blocking=True), device=dev)
            r = one_step(k, True, medium=m2, host=True)
            out = (r.iq.cpu(), r.residual.cpu(), r.status.cpu(), r.iterations.cpu())
            h2d = 3 * n * 4 + 2 * SYSTEMS_PER_STEP * 8
            d2h = sum(t.numel() * t.element_size() for t in out)
        e1.record(stream)
        barrier()
        e2e_ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
        e2e_value = solves / (float(e2e_ms) / 1e3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, wall, nsolves, _ = cpu_sample(args.cpu_sample_bins, 1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{args.cpu_sample_bins} bin(s) x 11 angles: assemble + SuperLU factor + solves, "
                         f"{wall:.1f} s on 1 core"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": L["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64/f64", "data": "synthetic",
            "config": {"workload": "breast record 1024x768 nodes dx=0.05mm, 11 angles x 294 bins "
                                   "(3234 systems); BiCGSTAB to true rel-res 1e-6 with the trained learned "
                                   "preconditioner (network set-up of each step's bins timed); plain Krylov "
                                   "(fixed shifted-Laplace, shift 0.15) under plain_krylov",
                       "systems_per_step": SYSTEMS_PER_STEP, "n_slots": N_SLOTS, "grid_zx": [rec.nz, rec.nx],
                       "l2": f"inputs larger than L2: {slots * n * 96 / 1e9:.2f} GB resident Krylov state per GPU",
                       "parallelism": f"frequency-sharded x{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "iteration_achieved": L["iteration_achieved"],
                         "iteration_frac": L["iteration_achieved"] / peak,
                         "kernel_ms": L["kms"]},
            "cpu_baseline": cpu,
            "clocks": clock_info,
            "solves": L["solves"],
            "plain_krylov": None if P is None else {
                "value": P["value"], "unit": UNIT, "ms_per_step": P["ms_per_step"], "solves": P["solves"],
                "learned_speedup": value / P["value"],
                "roofline": {"kernel": P["dominant"], "achieved": P["achieved"], "frac": P["achieved"] / peak,
                             "iteration_frac": P["iteration_achieved"] / peak, "kernel_ms": P["kms"],
                             "traffic": plain_traffic}},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
