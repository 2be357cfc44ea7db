#!/usr/bin/env python
"""Benchmark of the pm3d particle-mesh step on B200: PM particle-steps/s of the batched
ensemble (64 peaks, meshes 32^3..256^3, one graph replay per step), with the plain single-run
path on the same peaks, per-kernel HBM roofline, an end-to-end job through the public API,
and the CPU reference timed on the host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload batched|plain256|plain512]
    python bench.py --impl reference ...      # the reference algorithm on the host cores

One JSON line on stdout (rank 0).  Multi-GPU runs (torchrun) give every rank its own
ensemble (independent peaks, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import queue
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "PM particle-steps/s batched vs plain on 1 B200 at FP64-oracle tol; p50/p99 latency"
UNIT = "particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batched", "plain256", "plain512"], default="batched")
    ap.add_argument("--npeaks", type=int, default=64)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-errors", action="store_true", help="skip the per-output errors against the float64 oracle")
    ap.add_argument("--no-late", action="store_true", help="skip the device-timed window late in the run")
    ap.add_argument("--full-sort", action="store_true", help="re-sort every super-tile by cell every step (by default never)")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream latency run")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="arrival window of the served stream")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="mean request arrivals per second")
    ap.add_argument("--cpu-seconds", type=float, default=None,
                    help="timed window of the CPU sample (default 30 s for --impl reference, 10 s for cpu_baseline)")
    ap.add_argument("--tiles", default="auto", help="super-tile side: 'auto' (autotuned per mesh size) or 4/8/16")
    ap.add_argument("--fft", choices=["cufft", "native"], default="native",
                    help="64^3-512^3 transforms: cuFFT, or the native kernels with the Green multiply fused")
    return ap.parse_args()


# ------------------------------------------------------------------------------ workloads
def workload_specs(name: str, npeaks: int, seed: int, rank: int):
    from pbh_b200 import recipe
    if name == "batched":
        specs = recipe.ensemble(npeaks=npeaks, steps=150, seed=seed + 1000 * rank)
        desc = {"workload": f"batched ensemble: {npeaks} peaks, meshes from {{32,64,128,256}}^3 with particles = "
                            "cells, e~U[0,0.3], p~U[-0.1,0.1], delta0 log-uniform over collapse a in [0.3,1], "
                            "150 KDK steps over a_cfg 0.01..1, seeded k^-2 noise"}
    elif name == "plain256":
        specs = [recipe.single_peak(N=256, steps=200, seed=seed + rank)]
        desc = {"workload": "plain single run: 256^3 mesh, 256^3 particles, R=(0.10,0.09,0.08)L, "
                            "collapse of the first axis at a_cfg=0.8, 200 steps"}
    else:
        specs = [recipe.large_peak(N=512, steps=300, seed=seed + rank)]
        desc = {"workload": "large single run: 512^3 mesh and particles, e=0.3, p=0.1, collapse a_cfg=0.5, 300 steps"}
    return specs, desc


def workload_config(desc: dict, specs, gpus: int) -> dict:
    """The `config` of both arms: the workload only (its engine settings go under `engine`)."""
    return dict(desc, particles_per_gpu=int(sum(s.n for s in specs)), peaks=len(specs),
                l2="inputs larger than L2 (126 MB)", parallelism=f"replicas x{gpus}")


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------ CPU side
CPU_BYTES_PER_PARTICLE = 400      # resident set of one float64 oracle peak (6.1 GB measured at 256^3)
CPU_BYTES_PER_WORKER = 300 << 20   # interpreter, numpy and the oracle module


def _cpu_worker(args):
    """One peak of the recipe on the CPU oracle (float64 numpy restatement of pm3d): IC, the
    initial forces and `warmup` steps untimed; then, once every worker is ready (`barrier`),
    timed KDK steps until `budget` seconds have passed (at least `min_steps`).  Puts (index, N,
    particles * steps, seconds) on `out`, or (index, N, 0, error text)."""
    idx, N, R, delta0, seed, ratio, warmup, budget, min_steps, barrier, out = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    try:
        import warnings
        warnings.filterwarnings("ignore")
        from oracle import pm3d_oracle as O
        from oracle.recipe_oracle import recipe_ic
        mesh = O.Mesh(N, 1.0, N)
        ic = recipe_ic(mesh, R, delta0, 0.01, seed)
        tr = O.Trajectory(mesh, ic["x"], ic["p"])
        a = 1.0
        tr.acc, _d = O.accelerations(mesh, tr.x, a)   # what the first step would compute twice
        tr.acc_a = a
        for _ in range(warmup):
            a, _d = tr.step(a, a * ratio)
        try:
            barrier.wait(timeout=900)
        except threading.BrokenBarrierError:   # a worker failed: time this one all the same
            pass
        t0 = time.perf_counter()
        steps = 0
        while steps < min_steps or time.perf_counter() - t0 < budget:
            a, _d = tr.step(a, a * ratio)
            steps += 1
        out.put((idx, N, N ** 3 * steps, time.perf_counter() - t0))
    except Exception as exc:  # reported by the parent; the other workers carry on
        try:
            barrier.abort()
        except Exception:
            pass
        out.put((idx, N, 0, f"{type(exc).__name__}: {exc}"))


def allocate_cpu_workers(particles_by_mesh: dict, cores: int, mem_bytes: float) -> dict:
    """Workers per mesh size for the CPU sample of a mix: one per mesh size (largest meshes first
    when there are fewer cores than sizes), the rest in proportion to each size's particles (its
    share of the mix's work, so the cores are loaded roughly as a run of the whole mix would load
    them), within `mem_bytes` of host memory.  A size whose one worker does not fit is left out."""
    need = {N: CPU_BYTES_PER_PARTICLE * N ** 3 + CPU_BYTES_PER_WORKER for N in particles_by_mesh}
    alloc, used = {}, 0.0
    for N in sorted(particles_by_mesh, reverse=True):
        if len(alloc) < cores and used + need[N] <= mem_bytes:
            alloc[N] = 1
            used += need[N]
    total = sum(particles_by_mesh[N] for N in alloc)
    while sum(alloc.values()) < cores and alloc:
        # the size furthest below its share of the workers that still fits
        cands = [N for N in alloc if used + need[N] <= mem_bytes]
        if not cands:
            break
        N = max(cands, key=lambda m: particles_by_mesh[m] / total * cores - alloc[m])
        alloc[N] += 1
        used += need[N]
    return alloc


def host_memory_available() -> float:
    """Bytes this process can still use: the host's available memory, or less when a control
    group limits the container (its limit minus its current use)."""
    try:
        import psutil
        avail = float(psutil.virtual_memory().available)
    except Exception:
        avail = float(os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES"))
    for lim, cur in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            text = Path(lim).read_text().strip()
            if text != "max":
                avail = min(avail, float(text) - float(Path(cur).read_text().strip()))
            break
        except (OSError, ValueError):
            continue
    return max(avail, 0.0)


def mix_rate(particles_by_mesh: dict, rate_by_mesh: dict, cores: int) -> float:
    """Particle-steps/s of a whole mix of peaks on `cores` cores, each core running one peak at a
    time and none idle: one step of every peak costs sum_N P_N / r_N core-seconds (P_N the mix's
    particles on N^3 meshes, r_N one core's particle-steps/s on such a peak)."""
    return cores * sum(particles_by_mesh.values()) / sum(p / rate_by_mesh[N] for N, p in particles_by_mesh.items())


def cpu_rate(specs, budget: float, warmup: int, workers: int | None = None) -> dict:
    """The oracle port of the reference path on the host cores, one peak per worker process
    (spawned), the reference's own pattern for many runs (pbhgr/pbhgr/scan.py:223-232).  Every
    mesh size of the workload is sampled, all workers step at once over the same timed window,
    and the whole mix's rate follows from the per-size rates (`mix_rate`)."""
    import multiprocessing as mp
    import platform
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    workers = workers or cores
    pmesh = {}
    for s in specs:
        pmesh[s.N] = pmesh.get(s.N, 0) + s.n
    alloc = allocate_cpu_workers(pmesh, workers, 0.6 * host_memory_available())
    by_mesh = {}
    for s in specs:
        by_mesh.setdefault(s.N, []).append(s)
    picks = [by_mesh[N][i % len(by_mesh[N])] for N in sorted(alloc) for i in range(alloc[N])]
    ctx = mp.get_context("spawn")
    barrier, out = ctx.Barrier(len(picks)), ctx.Queue()
    procs = []
    for i, s in enumerate(picks):
        w = min(warmup, 1) if s.N <= 128 else 0   # numpy needs no warm-up beyond the initial forces
        task = (i, s.N, tuple(s.R), s.delta0, s.seed, s.ratio(), w, budget, 1, barrier, out)
        procs.append(ctx.Process(target=_cpu_worker, args=(task,), daemon=True))
    t0 = time.perf_counter()
    for p in procs:
        p.start()
    res, errors = [], []
    pending = set(range(len(procs)))
    while pending and time.perf_counter() - t0 < 1800:
        try:
            idx, N, ps, t = out.get(timeout=1.0)
        except queue.Empty:
            for i in sorted(pending):
                if procs[i].exitcode not in (None, 0):   # ended without reporting (killed)
                    pending.discard(i)
                    errors.append(f"{picks[i].N}^3: worker exit code {procs[i].exitcode}")
                    barrier.abort()
            continue
        pending.discard(idx)
        if ps:
            res.append((N, ps, t))
        else:
            errors.append(f"{N}^3: {t}")
    errors += [f"{picks[i].N}^3: no report" for i in sorted(pending)]
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.terminate()
    wall = time.perf_counter() - t0
    rates = {}
    for N, ps, t in res:
        rates.setdefault(N, []).append(ps / t)
    rate_by_mesh = {N: statistics.mean(v) for N, v in rates.items()}
    if not rate_by_mesh:
        raise RuntimeError("CPU sample failed: " + "; ".join(errors))
    # A mesh size without a measurement (it did not fit the host's memory) takes the rate of
    # the nearest measured size.
    full = {N: rate_by_mesh.get(N) or rate_by_mesh[min(rate_by_mesh, key=lambda m: abs(m - N))] for N in pmesh}
    value = mix_rate(pmesh, full, len(res))
    missing = sorted(set(pmesh) - set(rate_by_mesh))
    return {"value": value, "unit": UNIT, "cores": len(res), "kind": "port",
            "sample": f"{len(res)} peaks of the workload at once (one per core: "
                      + ", ".join(f"{alloc[N]} of {N}^3" for N in sorted(alloc))
                      + f"), float64 numpy restatement of pm3d, timed KDK steps over a common window of "
                      f"at least {budget:g} s after the IC and initial forces; the value is the whole "
                      f"{len(specs)}-peak mix on {len(res)} cores with no core idle, from the per-size "
                      f"per-core rates"
                      + (f"; meshes {missing}^3 took the nearest measured size's rate (host memory)" if missing else ""),
            "per_core_rate_by_mesh": {str(N): rate_by_mesh[N] for N in sorted(rate_by_mesh)},
            "errors": errors or None,
            "host_cpus": cores, "cpu": platform.processor() or platform.machine(), "wall_s": wall}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    specs, desc = workload_specs(args.workload, args.npeaks, args.seed, 0)
    cb = cpu_rate(specs, budget=30.0 if args.cpu_seconds is None else args.cpu_seconds, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (recipe peaks, seeded numpy noise)",
            "config": workload_config(desc, specs, args.gpus),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "per_core_rate_by_mesh")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------ GPU side
# Algorithmic bytes per launch of each kernel phase: n particles, N^3 cells,
# M modes; fc/hc: face and halo partials.
def algorithmic_bytes(phase: str, n: int, cells: int, modes: int, npass: int) -> float:
    if phase == "push":        # read state 32, write state 32, force grids 12 per cell
        return n * (32 + 32) + cells * 12.0
    if phase == "refresh":     # super-tile re-sort (only with --full-sort): read + write state
        return n * 64.0
    if phase == "deposit":     # read positions 16, write delta 4 per cell (face/halo partials are overhead)
        return n * 16.0 + cells * 4.0
    if phase == "green":       # read the spectrum 8, write three gradient spectra 24 per mode
        return modes * 32.0
    return 0.0


PHASES = ["push", "advance", "regroup", "refresh", "deposit", "r2c", "green", "c2r"]
NATIVE_FFT_SIZES = (64, 128, 256, 512)   # meshes the native transform serves (the others use cuFFT)


def launches_per_step(sizes, fft: str) -> int:
    """Our kernel launches in one steady (non-priming) step of an ensemble with these mesh sizes:
    push, energy, advance, bin layout and 2 relayout copies (gated: they return at once unless a
    push overflowed a bin), super-tile sort, deposit, fix-up and Green (10); the native
    transform adds 6 per mesh size it serves (3 passes each way) and drops the Green launch when
    it serves every mesh.  The radix sort runs only in steps that prime a peak."""
    native = {n for n in sizes if fft == "native" and n in NATIVE_FFT_SIZES}
    return 10 + 6 * len(native) - (1 if native and all(n in native for n in sizes) else 0)

# DRAM bytes (read + write) per launch from single-kernel ncu captures of the plain 256^3 run
# (the Green kernel's from the same run with cuFFT transforms), per particle (per mode for Green),
# scaled to a launch by the particles (modes) it processes; deposit includes its face fix-up.
NCU_TRAFFIC = {"push": 77.10, "deposit": 26.94, "green_per_mode": 25.89}


def replica_throughput(t_local: float, n_local: int, steps: int, dist=None, device="cpu"):
    """Whole-job particle-steps/s of independent replicas (one ensemble per rank, the same
    particle count on every rank): the job takes the slowest rank's device time.
    Returns (max time over ranks, value)."""
    import torch
    world = 1
    t = t_local
    if dist is not None:
        world = dist.get_world_size()
        tt = torch.tensor([t_local], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    return t, world * n_local * steps / t


def oracle_errors(specs, tiles, device: int, nsteps: int = 50) -> dict:
    """Per-output errors of the engine against the float64 oracle -- the checker, run outside
    every timed region.  For one seeded peak of each mesh size of the workload: nsteps KDK
    steps of the peak's own schedule from the engine's loaded particles, on the engine and on
    the float64 torch restatement of pm3d (oracle/pm3d_torch64.py, pinned to the numpy oracle);
    positions after nsteps (max, in cells), then the oracle's density and forces at the
    engine's final positions (relative L2).  Tolerances: density 1e-6, forces 1e-5, positions
    1e-5 cell."""
    import torch

    from oracle.pm3d_torch64 import TorchMesh, TorchTrajectory
    from pbh_b200 import _lib
    from pbh_b200.engine import Engine, PeakConfig
    from pbh_b200.ic import recipe_particles
    out = {}
    for N in sorted({s.N for s in specs}):
        sp = next(s for s in specs if s.N == N)
        eng = Engine([PeakConfig(N=N, Np=N, L=sp.L, tile=int(tiles.get(N, 0)))], device=device)
        x, p = recipe_particles(sp, device=device)
        eng.set_particles(0, x, p, 1.0, mode=_lib.SCHED_RATIO, param=sp.ratio(), max_steps=nsteps)
        del x, p
        x0, p0 = eng.particles(0)
        eng.run(nsteps + 2)
        c = eng.clock(0)
        x = eng.particles(0)[0]
        delta = eng.delta(0).double()
        acc = eng.acc(0, c.a)
        eng.close()
        tm = TorchMesh(N, sp.L, N, device=f"cuda:{device}")
        acc_ref, delta_ref = tm.forces(x, c.a)
        rel = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        e = {"density_rel_l2": rel(delta, delta_ref), "forces_rel_l2": rel(acc, acc_ref)}
        del acc_ref, delta_ref, acc, delta
        tr = TorchTrajectory(tm, x0, p0)
        a = 1.0
        for _ in range(nsteps):
            a, _ = tr.step(a, a * sp.ratio())
        d = x - tr.x
        d = d - sp.L * torch.round(d / sp.L)
        e["positions_cells"] = float(d.abs().max()) / tm.dx
        e["seed"] = sp.seed
        out[str(N)] = e
        del tr, x, x0, p0, tm
        torch.cuda.empty_cache()
    worst = {k: max(v[k] for v in out.values()) for k in ("density_rel_l2", "forces_rel_l2", "positions_cells")}
    return {"vs": "float64 pm3d restatement on the same initial particles (same positions for density and forces)",
            "steps": nsteps, "by_mesh": out, "max": worst,
            "tolerance": {"density_rel_l2": 1e-6, "forces_rel_l2": 1e-5, "positions_cells": 1e-5},
            "within": bool(worst["density_rel_l2"] <= 1e-6 and worst["forces_rel_l2"] <= 1e-5
                           and worst["positions_cells"] <= 1e-5)}


# Ideal HBM bytes of a whole step: 112 per particle outside the transforms (push 64 + 12 per cell
# of force grids, deposit 16 + 4 per cell, Green 32 per mode = 16 per cell; particles = cells) and
# 24 per cell for the transforms (R2C reads delta and writes the half spectrum, C2R reads it and
# writes three force grids).
IDEAL_BYTES_PER_PARTICLE = 112.0
IDEAL_FFT_BYTES_PER_CELL = 24.0


def run_ours(args):
    import numpy as np
    import torch

    from pbh_b200 import _lib
    from pbh_b200.batch import Ensemble, plain_rate, pm3d_step_rate

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    specs, desc = workload_specs(args.workload, args.npeaks, args.seed, rank)
    need = 1 + args.warmup + args.steps
    if need > min(s.steps for s in specs):
        raise SystemExit(f"warmup + steps ({need}) exceed the run length ({min(s.steps for s in specs)})")
    if args.tiles == "auto":
        from pbh_b200.tune import autotune
        tiles = autotune({s.N for s in specs} | ({64, 128, 256} if not args.no_serve else set()), device=local)
    else:
        tiles = {s.N: min(int(args.tiles), s.N) for s in specs}
    ens = Ensemble(specs, device=local, bucket_sort=not args.full_sort, tiles=tiles, native_fft=args.fft == "native")

    lib = _lib.load()
    info = (np.zeros(6, dtype=np.int64))
    lib.pm_engine_info(ens.engine._h, info.ctypes.data)
    npass = int(info[3])
    ens.load()
    ens.step(1 + args.warmup)                     # prime + warm-up steps
    stream = torch.cuda.ExternalStream(lib.pm_engine_stream(ens.engine._h), device=local)
    n_step = ens.active_particles()
    assert n_step == ens.n_particles, "every peak must be stepping during the timed region"
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ens.engine.sync()
    relayouts0 = sum(s.relayouts for s in ens.stats())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    e0.record(stream)
    ens.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    t, value = replica_throughput(e0.elapsed_time(e1) / 1e3, n_step, args.steps, dist,
                                  device=f"cuda:{local}")
    ms_per_step = t / args.steps * 1e3
    relayouts = sum(s.relayouts for s in ens.stats()) - relayouts0

    # Per-kernel device times: a few ungraphed steps with events between phases, same stream.
    ph = ens.timed_phases(16)                     # sixteen steady steps
    # A second device-timed window late in the run (past the collapse of the early peaks).
    late = None
    run_len = min(sp.steps for sp in specs)
    done_steps = args.warmup + args.steps + 16
    if run_len >= 140 and done_steps <= 120 and not args.no_late:
        ens.step(120 - done_steps)
        n_late = ens.active_particles()
        ens.engine.sync()
        r_late0 = sum(s.relayouts for s in ens.stats())
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        ens.step(20)
        l1.record(stream)
        l1.synchronize()
        t_late = l0.elapsed_time(l1) / 1e3
        a_cfg = ens.clocks()[0].a / 100.0
        r_late = sum(s.relayouts for s in ens.stats()) - r_late0
        late = {"steps": [121, 140], "ms_per_step": t_late / 20 * 1e3, "value": n_late * 20 / t_late, "unit": UNIT,
                "relayouts": r_late,
                "a_cfg_end": a_cfg,
                "peaks_past_design_collapse": int(sum(1 for sp in specs if sp.a_collapse_cfg <= a_cfg))}
        # Where the late steps spend their time: per-phase device ms over the next 4 (ungraphed) steps.
        ph_late = ens.timed_phases(4)
        late["phase_ms"] = {name: round(float(v), 4) for name, v in zip(PHASES, ph_late)}
    cells = sum(s.N ** 3 for s in specs)
    # modes the Green kernel handles (the native 256^3 transform applies its own multiply)
    modes = sum(s.N * s.N * (s.N // 2 + 1) for s in specs if not (args.fft == "native" and s.N in NATIVE_FFT_SIZES))
    kern = {}
    for k, name in enumerate(PHASES):
        b = algorithmic_bytes(name, n_step, cells, modes, npass)
        if name == "refresh" and not args.full_sort:
            b = 0.0                                # no re-sort in these steps
        kern[name] = {"ms": ph[k], "algorithmic_bytes": b, "gbs": (b / (ph[k] / 1e3) / 1e9) if b and ph[k] > 0 else None}
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    if peaks_file.exists():
        hbm = float(json.loads(peaks_file.read_text())["hbm_gbs"])
        hbm_src = "measured"
    else:
        hbm, hbm_src = 6650.0, "fallback"
    ours = {k: v for k, v in kern.items() if k in ("push", "refresh", "deposit", "green") and v["gbs"] is not None}
    top = max(ours, key=lambda k: ours[k]["ms"])
    def traffic(name):
        if name == "green":
            return NCU_TRAFFIC["green_per_mode"] * modes
        return NCU_TRAFFIC[name] * n_step if name in NCU_TRAFFIC else None
    roofline = {"bound": "hbm", "kernel": top, "achieved": kern[top]["gbs"], "peak": hbm, "unit": "GB/s",
                "frac": kern[top]["gbs"] / hbm, "traffic": traffic(top),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of single-kernel captures of the "
                                  "plain 256^3 run, per particle, times this launch's particles",
                "algorithmic_bytes": kern[top]["algorithmic_bytes"], "peak_source": hbm_src,
                "per_kernel": {k: {"ms": round(v["ms"], 4), "gbs": None if v["gbs"] is None else round(v["gbs"], 1),
                                   "frac": None if v["gbs"] is None else round(v["gbs"] / hbm, 3)}
                               for k, v in kern.items()},
                "fft_ms": round(ph[5] + ph[7], 4), "step_ms_ungraphed": round(float(ph.sum()), 4)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (fields, offsets, momenta; i32 cells; i64 fixed-point density sums)",
            "data": "synthetic (recipe peaks, seeded numpy noise)",
            "config": workload_config(desc, specs, world),
            "engine": {"regroup": "push into bins, super-tile re-sort every step" if args.full_sort else
                       "push into bins, no super-tile re-sort", "timed_steps": [1 + args.warmup,
                                                                                       args.warmup + args.steps],
                       "super_tiles": {str(k): v for k, v in sorted(tiles.items())},
                       "relayouts_timed": relayouts,
                       "fft_64_to_512": "native (Green fused into the inverse)" if args.fft == "native" else "cuFFT"},
            "clocks": clocks, "gpu_launches": args.steps * launches_per_step([sp.N for sp in specs], args.fft),
            "roofline": roofline}
    if late is not None:
        line["late_window"] = late

    if rank == 0 and not args.no_plain and args.workload == "batched":
        pr = plain_rate(specs, steps=8, warmup=3, device=local, tiles=tiles)
        # Upper bound of batched/plain: the plain runs' summed step time over the time of the
        # whole ensemble's step at the HBM roofline (every byte moved once at the measured peak).
        plain_ms = sum(pr["step_s_by_mesh"][str(sp.N)] for sp in specs) * 1e3
        ideal_ms = sum(IDEAL_BYTES_PER_PARTICLE * sp.n + IDEAL_FFT_BYTES_PER_CELL * sp.N ** 3
                       for sp in specs) / (hbm * 1e9) * 1e3
        line["plain"] = dict(pr, batched_over_plain=value / world / pr["particle_steps_per_s"],
                             how="each peak alone in a single-peak engine, sequentially, same kernels",
                             bound={"plain_ms_per_ensemble_step": plain_ms, "roofline_ms_per_ensemble_step": ideal_ms,
                                    "batched_ms_per_step": ms_per_step,
                                    "max_batched_over_plain": plain_ms / ideal_ms,
                                    "how": "sum of the plain per-peak step times / the ensemble step at the HBM "
                                           "roofline (112 B per particle + 24 B per cell at the measured peak)"})
        ps = pm3d_step_rate(specs, steps=5, warmup=2, device=local)
        line["plain_pm3d_step"] = dict(ps, batched_over_pm3d_step=value / world / ps["particle_steps_per_s"],
                                       how="each peak alone through PM3D.step (delta returned to the host "
                                           "every step, as the reference driver uses it); wall clock")

    if not args.no_e2e:
        line["e2e"] = e2e_job(ens, specs, torch, local)
    ens.close()
    del ens
    if rank == 0 and not args.no_errors:
        line["errors"] = oracle_errors(specs, tiles, local)
    if rank == 0 and not args.no_serve:
        line["served"] = served_stream(args, local, tiles)
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_rate(specs, budget=10.0 if args.cpu_seconds is None else args.cpu_seconds, warmup=1)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "per_core_rate_by_mesh")}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def e2e_job(ens, specs, torch, device):
    """The whole job through the public batch API: per-peak noise fields start in pinned host
    memory, are copied to the device, turned into particles (device IC), then every step runs
    with its per-peak statistics read back to the host, and at the end every peak's final
    density grid comes back to the host (the job's result)."""
    import ctypes

    import numpy as np

    from pbh_b200 import _lib
    noises = []
    for s in specs:
        h = torch.empty((s.N,) * 3, dtype=torch.float64).pin_memory()
        h.numpy()[...] = np.random.default_rng(s.seed).standard_normal((s.N,) * 3)
        noises.append(h)
    h2d = sum(int(h.numel()) * 8 for h in noises)
    results = ens.result_buffers()              # page-locked result buffers, allocated once like the inputs
    steps = min(s.steps for s in specs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ens.load(noises=noises)
    torch.cuda.synchronize()
    t_load = time.perf_counter()
    stats_bytes = 0
    done = 0
    for _ in range(steps + 2):                   # prime + steps + closing kick
        ens.step(1)
        st = ens.stats()
        stats_bytes += len(st) * ctypes.sizeof(_lib.StatsInfo)
        done += 1
    t_steps = time.perf_counter()
    finals = ens.deltas(results)                 # the job's result: every peak's final delta
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    relayouts = sum(s.relayouts for s in ens.stats())
    del noises
    result_bytes = sum(int(f.nbytes) for f in finals)
    assert all(np.isfinite(f).all() for f in finals)
    ps = sum(s.n for s in specs) * steps
    return {"value": ps / t, "unit": UNIT, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": (stats_bytes + result_bytes) / steps,
            "job_steps": steps, "seconds": t, "result_bytes": result_bytes, "relayouts": relayouts,
            "seconds_by_part": {"load": round(t_load - t0, 4), "steps": round(t_steps - t_load, 4),
                                "result": round(t0 + t - t_steps, 4)},
            "how": "public Ensemble API: pinned host noise -> device IC -> all steps with per-step stats to the "
                   "host -> every peak's final delta to the host; wall clock"}


def served_stream(args, device, tiles=None):
    """The served form: Poisson arrivals of single-peak collapse runs (meshes 64^3-256^3,
    (e, p, delta0) as the ensemble) admitted into a slot pool under a 150 GB HBM budget,
    continuously batched, each run ending at its collapse (max delta >= 50) or last step."""
    import numpy as np

    from pbh_b200.serve import Server, ServerConfig, latency_summary, poisson_arrivals
    arrivals = poisson_arrivals(rate=args.serve_rate, duration=args.serve_seconds, seed=args.seed, steps=150)
    cfg = ServerConfig(slots={64: 32, 128: 32, 256: 24}, budget_bytes=150e9, delta_collapse=50.0, keep_delta=True,
                       device=device, tiles=tiles)
    srv = Server(cfg)
    t0 = time.perf_counter()
    done = srv.serve(arrivals, timeout=args.serve_seconds + 240.0)
    wall = time.perf_counter() - t0
    out = latency_summary(done)
    out.update(requests=len(arrivals), rate_per_s=args.serve_rate, arrival_window_s=args.serve_seconds,
               wall_s=wall, particle_steps_per_s=srv.particle_steps / wall, engine_steps=srv.engine_steps,
               collapsed=int(sum(1 for r in done if r.a_collapse_cfg > 0)),
               mean_steps=float(np.mean([r.steps for r in done])) if done else None,
               slots={str(k): v for k, v in cfg.slots.items()}, budget_gb=cfg.budget_bytes / 1e9,
               device_gb=srv.engine.device_bytes / 1e9,
               how="latency = arrival to result (collapse a, final delta) on the host; wall-clock")
    srv.close()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
