"""Throughput of the batched frequency-domain Helmholtz solve on B200.

Workload: the synthetic breast record, 1024 (x) x 768 (z) nodes at 0.05 mm,
11 plane-wave angles x 294 frequency bins (4.015-8.896 MHz) = 3234 systems,
BiCGSTAB to a true relative residual of 1e-6.  One step solves a batch of
SYSTEMS_PER_STEP systems (4 bins x 11 angles) through the resident-slot queue;
a rank's bins come from the longest-first partition of the band over the ranks
(``nsrno_b200.shard.partition_bins``), visited by a fixed stride so that every
step sees low and high frequencies.  Under torchrun every rank takes different
bins (weak scaling, no collective on the data path).

Two arms run on the same GPU and the same steps: the headline "learned-init"
arm (the trained learned preconditioner: its network set-up for the step's
bins is inside the timed region) and the "plain Krylov" arm (the fixed
shifted-Laplace preconditioner, shift 0.15), reported under ``plain_krylov``.
Before timing, the launch shapes of both arms are chosen by the autotuner
(``nsrno_b200.tune``; cached per GPU and grid).  Per-kernel durations come from
a separate, untimed profiling pass.  ``record`` pushes all 3234 systems of the
record through one solve queue (learned arm; ``--record`` adds the plain arm).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--record]

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import platform
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
    p.add_argument("--no-tune", action="store_true", help="use the built-in launch shapes")
    p.add_argument("--retune", action="store_true", help="tune even when a cached choice exists")
    p.add_argument("--record", action="store_true", help="also run the plain arm over the whole record")
    p.add_argument("--no-record", action="store_true", help="skip the whole-record run")
    p.add_argument("--host-loop", action="store_true",
                   help="host-polled solve loop (every kernel a separate launch, for a profiler's launch list)")
    p.add_argument("--plain-only", action="store_true",
                   help="run only the plain-Krylov arm (for profiling it); prints a short line, not the bench line")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _coprime_stride(n, target):
    s = max(1, int(round(target)))
    while math.gcd(s, n) != 1:
        s += 1
    return s


def rank_bins(record, rank, world):
    """This rank's bins (longest-first partition of the band), in a stride
    order that spreads consecutive steps over the whole band."""
    from nsrno_b200.shard import partition_bins
    mine = partition_bins(record.frequencies, world)[rank]
    n = len(mine)
    order = (np.arange(n) * _coprime_stride(n, 0.514 * n)) % n
    return mine[order]


def step_systems(record, step, rank, world):
    """(freqs, angles) of one step on one rank, highest frequency first."""
    mine = rank_bins(record, rank, world)
    first = step * BINS_PER_STEP
    bins = [mine[(first + k) % len(mine)] for k in range(BINS_PER_STEP)]
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


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


# ---------------------------------------------------------------------------
# CPU arm: the reference algorithm of the path (assemble, one SuperLU factor
# per frequency shared by all angles, solve) restated by the oracle.  Worker
# processes build the record once, outside any timed region.
# ---------------------------------------------------------------------------
_REC = None
_SPEC = None


def _cpu_init():
    os.environ["OMP_NUM_THREADS"] = "1"
    global _REC, _SPEC
    from oracle import helmholtz_ref as H
    from nsrno_b200.media import breast_record
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except ImportError:
        pass
    _REC = breast_record()
    r = _REC
    _SPEC = H.Spec(nz=r.nz, nx=r.nx, h=r.h, n_pml=r.n_pml, c0=r.c0, rho0=r.rho0, pml_strength=r.pml_strength,
                   face=r.face, rx_cols=r.rx_cols, aperture_half_width=r.aperture_half_width,
                   alpha_power=r.alpha_power)


def _cpu_one_bin(b):
    from oracle import helmholtz_ref as H
    rec = _REC
    fields, seconds, res = H.time_lu_frequency(_SPEC, rec.c, rec.rho, rec.alpha, rec.frequencies[b], rec.angles)
    return seconds, res, len(rec.angles)


def _noop(_):
    return os.getpid()


class CpuPool:
    """A warmed pool of `n` single-threaded worker processes (spawn)."""

    def __init__(self, n):
        import multiprocessing as mp
        self.n = n
        self.pool = None
        if n > 1:
            self.pool = mp.get_context("spawn").Pool(n, initializer=_cpu_init)
            self.pool.map(_noop, range(4 * n))
        else:
            _cpu_init()

    def bins(self, bins):
        t0 = time.perf_counter()
        out = self.pool.map(_cpu_one_bin, bins, chunksize=1) if self.pool else [_cpu_one_bin(b) for b in bins]
        wall = time.perf_counter() - t0
        return wall, sum(o[2] for o in out), max(o[1] for o in out)

    def close(self):
        if self.pool:
            self.pool.close()
            self.pool.join()


def _config1_gmres(args):
    """One config-1 system by the oracle's GMRES(30) to 1e-7 (nsrno/wave_solver.py:9-36 restated), 1 thread."""
    os.environ["OMP_NUM_THREADS"] = "1"
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except ImportError:
        pass
    from oracle import helmholtz_ref as H
    from nsrno_b200.media import blob_record
    s = args
    rec = blob_record()
    spec = H.Spec(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, c0=rec.c0, rho0=rec.rho0,
                  pml_strength=rec.pml_strength, face=rec.face, rx_cols=rec.rx_cols,
                  aperture_half_width=rec.aperture_half_width, alpha_power=rec.alpha_power)
    f, th = rec.systems()
    t0 = time.perf_counter()
    A = H.operator(spec, rec.c, rec.rho, rec.alpha, f[s]) * rec.h ** 2
    b = H.plane_wave_rhs(spec, f[s], th[s]) * rec.h ** 2
    kh2 = (2 * math.pi * f[s] / rec.c0 * rec.h) ** 2
    qz = np.sin(np.pi * np.arange(rec.nz) / rec.nz) ** 2
    qx = np.sin(np.pi * np.arange(rec.nx) / rec.nx) ** 2
    mul = 1.0 / (-4.0 * (qz[:, None] + qx[None, :]) + kh2 * (1 + 0.15j))
    pre = lambda v: np.fft.ifft2(np.fft.fft2(v.reshape(rec.nz, rec.nx)) * mul).ravel()
    x, reason, steps = H.gmres(lambda v: A @ v, b, restart=30, max_cycles=400, tolerance=1e-7, precondition=pre)
    return time.perf_counter() - t0, reason, steps


def config1_cpu(cores):
    """Config 1 (256x256 blobs, 6 systems) on the host: the oracle's SuperLU
    (one factorisation per frequency) and its GMRES(30) to 1e-7, at 1 thread
    and over all cores (one process per system)."""
    import multiprocessing as mp
    from oracle import helmholtz_ref as H
    from nsrno_b200.media import blob_record
    try:
        from threadpoolctl import threadpool_limits
        limit = threadpool_limits(1)
    except ImportError:
        limit = None
    rec = blob_record()
    spec = H.Spec(nz=rec.nz, nx=rec.nx, h=rec.h, n_pml=rec.n_pml, c0=rec.c0, rho0=rec.rho0,
                  pml_strength=rec.pml_strength, face=rec.face, rx_cols=rec.rx_cols,
                  aperture_half_width=rec.aperture_half_width, alpha_power=rec.alpha_power)
    t0 = time.perf_counter()
    for f in rec.frequencies:
        H.time_lu_frequency(spec, rec.c, rec.rho, rec.alpha, f, rec.angles)
    lu_s = time.perf_counter() - t0
    n_sys = len(rec.frequencies) * len(rec.angles)
    one = [_config1_gmres(s) for s in range(n_sys)]
    procs = max(1, min(cores, n_sys))
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(procs) as pool:
        par = pool.map(_config1_gmres, range(n_sys), chunksize=1)
    all_s = time.perf_counter() - t0
    if limit is not None:
        limit.restore_original_limits()
    return {"systems": n_sys, "superlu_1thread_solves_per_s": n_sys / lu_s,
            "gmres30_1thread_solves_per_s": n_sys / sum(o[0] for o in one),
            "gmres30_allcores_solves_per_s": n_sys / all_s, "gmres30_allcores_processes": procs,
            "gmres30_steps_mean": float(np.mean([o[2] for o in one])),
            "gmres30_converged": all(o[1] == "converged" for o in one) and all(o[1] == "converged" for o in par)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    from nsrno_b200.media import breast_record
    rec = breast_record()
    # every host core, bounded by memory (a SuperLU factorisation of the
    # 786,432-node system holds about 2 GB)
    try:
        import psutil
        by_mem = max(1, int(psutil.virtual_memory().available // (3 << 30)))
    except ImportError:
        by_mem = cores
    procs = max(1, min(cores, by_mem, len(rec.frequencies)))
    pool = CpuPool(procs)
    perm = rank_bins(rec, 0, 1)
    # each step: `procs` bins (11 angles each) over the warmed worker processes
    pos = 0
    for _ in range(min(args.warmup, 1)):
        pool.bins([int(perm[pos % len(perm)])])   # primes each worker's scipy state
        pos += 1
    t_total = 0.0
    solves_total = 0
    for _ in range(max(1, args.steps)):
        bins = [int(perm[(pos + k) % len(perm)]) for k in range(procs)]
        pos += procs
        wall, solves, res = pool.bins(bins)
        t_total += wall
        solves_total += solves
    pool.close()
    value = solves_total / t_total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "breast 1024x768 dx=0.05mm, 11 angles x 294 bins; CPU: assemble + SuperLU "
                                   "factor per bin + 11 angle solves (theranostic/wave.py:240-273 restated)",
                       "bins_per_step": procs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                             "host_cores": cores, "cpu_model": cpu_model(), "memory_bound_processes": by_mem,
                             "sample": f"{procs} bins x 11 angles per step on {procs} single-threaded processes "
                                       f"(pool and medium built outside the timed wall)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from nsrno_b200 import Geometry, Medium, Workspace, _lib, solve_batched, tune
    from nsrno_b200.solver import solve_progress
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

    # Launch shapes of both arms (autotuner, untimed; cached per GPU and grid).
    shapes = {True: ({}, 16), False: ({}, 16)}
    tuning = {}
    if not args.no_tune:
        f_s, a_s = step_systems(rec, 0, rank, world)
        sample_setup = net.setup(med, np.unique(f_s))
        for learned in (True, False):
            if learned is False and args.no_plain:
                continue
            r = tune.tuned_config(med, f_s, a_s, learned=sample_setup if learned else None, n_slots=N_SLOTS,
                                  refresh=args.retune, iterations=32, repeats=3)
            shapes[learned] = tune.split(r["config"])
            tuning["learned" if learned else "plain"] = {
                "config": r["config"], "cached": r["cached"], "us_per_system_iteration": 1e6 * r["cost_s"],
                "default_us_per_system_iteration": 1e6 * r["default_cost_s"], "gain": r["gain"]}
        del sample_setup

    def one_step(step, learned, medium=med, profile=0, host=False):
        f, a = step_systems(rec, step, rank, world)
        if host:
            f = torch.from_numpy(f).pin_memory().to(dev, non_blocking=True)
            a = torch.from_numpy(a).pin_memory().to(dev, non_blocking=True)
        setup = None
        if learned:
            setup = net.setup(medium, torch.unique(torch.as_tensor(f, device=dev)))
        tiles, k = shapes[learned]
        return solve_batched(medium, f, a, tolerance=TOL, max_iterations=MAX_ITERS, n_slots=N_SLOTS,
                             profile_iterations=profile, workspace=ws, learned=setup, tiles=tiles,
                             graph_iterations=k, blocking=True if args.host_loop else None)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    stream = torch.cuda.current_stream()

    def max_ms(ms):
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t)

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
            results.append(one_step(k, learned))
        t1.record(stream)
        barrier()
        clock_info = clocks.stop() if clocks else None
        return max_ms(t0.elapsed_time(t1)), results, clock_info

    def profiled(learned):
        """Per-kernel event durations of one step (untimed pass, launches not graphed)."""
        r = one_step(0, learned, profile=PROFILE_ITERS)
        torch.cuda.synchronize()
        return r.extra["stats"]["kernel_ms"]

    n = rec.nz * rec.nx
    slots = min(N_SLOTS, SYSTEMS_PER_STEP)
    peak, peak_kind = peak_hbm()
    solves = SYSTEMS_PER_STEP * args.steps * world

    def summarise(ms_max, results, kms, per_node):
        status = torch.cat([r.status for r in results]).cpu().numpy()
        iters = torch.cat([r.iterations for r in results]).cpu().numpy()
        resid = torch.cat([r.residual for r in results]).cpu().numpy()
        alg = {k: n * (per_node[k] * slots + COEF_BYTES.get(k, 0)) for k in per_node}
        dominant = max(kms, key=kms.get)
        iter_ms = sum(kms.values())
        return dict(value=solves / (ms_max / 1e3), ms_per_step=ms_max / max(1, args.steps), kms=kms, alg=alg,
                    dominant=dominant, achieved=alg[dominant] / (kms[dominant] / 1e3) / 1e9,
                    iteration_achieved=sum(alg.values()) / (iter_ms / 1e3) / 1e9,
                    launches=int(sum(solve_progress(r)[3] for r in results)),
                    solves={"total": int(len(status)), "converged": int((status == _lib.CONVERGED).sum()),
                            "iterations_mean": float(iters.mean()), "iterations_max": int(iters.max()),
                            "residual_max": float(resid.max())})

    if args.plain_only:
        ms_p, res_p, _ = timed(False)
        P = summarise(ms_p, res_p, profiled(False), KERNEL_BYTES)
        if rank == 0:
            print(json.dumps({"arm": "plain", "value": P["value"], "unit": UNIT, "kernel_ms": P["kms"],
                              "solves": P["solves"]}), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    ms_l, res_l, clock_info = timed(True, sample_clocks=True)
    P = None
    if not args.no_plain:
        ms_p, res_p, _ = timed(False)
    L = summarise(ms_l, res_l, profiled(True), LEARNED_BYTES)
    if not args.no_plain:
        P = summarise(ms_p, res_p, profiled(False), KERNEL_BYTES)
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
        e2e_value = solves / (max_ms(e0.elapsed_time(e1)) / 1e3)

    # The whole record through one queue: every system of this rank's bins.
    record = None
    if not args.no_record:
        mine = rank_bins(rec, rank, world)
        f_all = np.repeat(rec.frequencies[mine], N_ANGLES)
        a_all = np.tile(rec.angles, len(mine))
        order = np.argsort(-f_all, kind="stable")
        f_all, a_all = f_all[order], a_all[order]
        record = {"systems": int(len(f_all) * world), "bins": int(len(mine) * world)}
        for learned in ((True, False) if args.record and not args.no_plain else (True,)):
            barrier()
            r0 = torch.cuda.Event(enable_timing=True)
            r1 = torch.cuda.Event(enable_timing=True)
            r0.record(stream)
            setup = net.setup(med, np.unique(f_all)) if learned else None
            tiles, k = shapes[learned]
            res = solve_batched(med, f_all, a_all, tolerance=TOL, max_iterations=MAX_ITERS, n_slots=N_SLOTS,
                                workspace=ws, learned=setup, tiles=tiles, graph_iterations=k)
            r1.record(stream)
            barrier()
            ms = max_ms(r0.elapsed_time(r1))
            st = res.status.cpu().numpy()
            record["learned" if learned else "plain"] = {
                "value": len(f_all) * world / (ms / 1e3), "unit": UNIT, "seconds": ms / 1e3,
                "converged_on_rank0": int((st == _lib.CONVERGED).sum()), "systems_on_rank0": int(len(st)),
                "iterations_mean": float(res.iterations.float().mean()),
                "residual_max": float(res.residual.max())}
            del setup, res

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        pool = CpuPool(1)
        wall, nsolves, _ = pool.bins([int(b) for b in rank_bins(rec, 0, 1)[:args.cpu_sample_bins]])
        cpu = {"value": nsolves / wall, "unit": UNIT, "cores": 1, "kind": "port", "host_cores": cores,
               "cpu_model": cpu_model(),
               "sample": f"{args.cpu_sample_bins} bin(s) x 11 angles of the breast record: assemble + SuperLU "
                         f"factor + solves, {wall:.1f} s on 1 core",
               "config1": config1_cpu(cores)}

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
                       "parallelism": f"frequency-sharded x{world}",
                       "tiles": {"learned": shapes[True][0], "learned_graph_iterations": shapes[True][1],
                                 "plain": shapes[False][0], "plain_graph_iterations": shapes[False][1]}},
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
            "tuning": tuning or None,
            "record": record,
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
