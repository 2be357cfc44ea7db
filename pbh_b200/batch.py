"""Batched ensembles: many independent peaks of different mesh sizes resident on one GPU and
advanced together, one captured graph replay per step for the whole ensemble.

Each peak is one PM3D run of the recipe in ``pbh_b200.recipe`` (Gaussian peak + k^-2 noise,
``steps`` KDK steps uniform in ln a from a = 1 to 100).  The per-peak schedule, the pending
closing kick and collapse detection all live in device memory, so peaks can start and finish
on different steps without the host touching the graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .engine import Engine, PeakConfig
from .ic import recipe_particles


class Ensemble:
    def __init__(self, specs, device: int = 0, graph: bool = True, bucket_sort: bool = True, tiles=None,
                 delta_collapse: float = 0.0, native_fft: bool = True):
        self.specs = list(specs)
        if tiles == "auto":                      # per mesh size, timed on this GPU (pbh_b200.tune)
            from .tune import autotune
            tiles = autotune({sp.N for sp in self.specs}, device=device)
        tiles = tiles or {}
        self.tiles = {int(k): int(v) for k, v in tiles.items()}
        self.cfgs = [PeakConfig(N=s.N, Np=s.N, L=s.L, tile=int(tiles.get(s.N, 0))) for s in self.specs]
        self.engine = Engine(self.cfgs, device=device, bucket_sort=bucket_sort, graph=graph, native_fft=native_fft)
        self.device = device
        self.delta_collapse = float(delta_collapse)
        self.n = np.array([s.n for s in self.specs], dtype=np.int64)

    @property
    def n_particles(self) -> int:
        return int(self.n.sum())

    def load(self, peaks=None, noises=None):
        """Device initial conditions for the given peaks (all by default) and their schedules."""
        idx = range(len(self.specs)) if peaks is None else peaks
        for j, i in enumerate(idx):
            s = self.specs[i]
            x, p = recipe_particles(s, device=self.device, noise=None if noises is None else noises[j])
            self.engine.set_particles(i, x, p, 1.0, mode=_lib.SCHED_RATIO, param=s.ratio(), max_steps=s.steps)
            if self.delta_collapse > 0:
                _lib.load().pm_set_collapse_threshold(self.engine._h, i, self.delta_collapse, 0)
            del x, p

    def step(self, k: int = 1):
        self.engine.run(k)

    def clocks(self):
        arr = (_lib.ClockInfo * len(self.specs))()
        _lib.check(_lib.load().pm_get_clocks_all(self.engine._h, arr), "pm_get_clocks_all")
        return list(arr)

    def stats(self):
        arr = (_lib.StatsInfo * len(self.specs))()
        rc = _lib.load().pm_get_stats_all(self.engine._h, arr)
        _lib.check(rc, "pm_get_stats_all")
        return list(arr)

    def result_buffers(self):
        """Page-locked host buffers for deltas(), one N^3 float32 array per peak (allocate once
        and reuse: page-locking memory is slow)."""
        torch = _lib.require_cuda()
        return [torch.empty((s.N,) * 3, dtype=torch.float32, pin_memory=True) for s in self.specs]

    def deltas(self, out=None):
        """Every peak's density contrast of its last deposit (N^3 float32) on the host: one
        asynchronous copy per peak into page-locked memory behind the engine's work, then one
        wait.  `out`: buffers from result_buffers() (allocated here if None).  Returns a list of
        numpy arrays (views of the page-locked buffers)."""
        lib = _lib.load()
        bufs = out if out is not None else self.result_buffers()
        outs = []
        for i, s in enumerate(self.specs):
            buf = bufs[i]
            if tuple(buf.shape) != (s.N,) * 3 or not buf.is_pinned():
                raise ValueError(f"result buffer {i} must be a page-locked {s.N}^3 float32 tensor")
            _lib.check(lib.pm_get_delta_async(self.engine._h, i, buf.data_ptr()), "pm_get_delta_async")
            outs.append(buf)
        self.engine.sync()
        return [b.numpy() for b in outs]

    def active_particles(self) -> int:
        return int(sum(n for n, c in zip(self.n, self.clocks()) if c.state == _lib.STATE_RUN))

    def run_to_end(self, chunk: int = 16):
        """Replay until every peak is idle; returns the number of engine steps."""
        steps = 0
        while True:
            cl = self.clocks()
            if all(c.state == _lib.STATE_IDLE for c in cl):
                return steps
            self.engine.run(chunk)
            steps += chunk

    def timed_phases(self, nsteps: int):
        """Per-phase device ms (push, energy + advance, regroup (priming sort, relayouts),
        refresh (super-tile re-sort), deposit with its face fix-up, R2C, Green, C2R) over nsteps
        ungraphed steps, from CUDA events on the engine's stream."""
        ms = (ctypes.c_double * 8)()
        _lib.check(_lib.load().pm_run_timed(self.engine._h, int(nsteps), ms), "pm_run_timed")
        return np.array(list(ms)) / max(nsteps, 1)

    def close(self):
        self.engine.close()


def plain_rate(specs, steps: int = 8, warmup: int = 3, device: int = 0, tiles=None) -> dict:
    """The plain single-run path on the same work: every peak alone in its own single-peak
    engine (graph-captured), one after another.  Returns particle-steps/s over the ensemble."""
    torch = _lib.require_cuda()
    by_n = {}
    for s in specs:
        by_n.setdefault(s.N, []).append(s)
    total_ps, total_t = 0.0, 0.0
    per = {}
    for N, group in sorted(by_n.items()):
        s = group[0]
        ens = Ensemble([s], device=device, tiles=tiles)
        ens.load()
        ens.step(1 + warmup)
        stream = torch.cuda.ExternalStream(_lib.load().pm_engine_stream(ens.engine._h))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ens.engine.sync()
        e0.record(stream)
        ens.step(steps)
        e1.record(stream)
        e1.synchronize()
        t_step = e0.elapsed_time(e1) / 1e3 / steps
        per[N] = t_step
        total_ps += len(group) * s.n
        total_t += len(group) * t_step
        ens.close()
    return {"particle_steps_per_s": total_ps / total_t, "step_s_by_mesh": {str(k): v for k, v in per.items()}}


def pm3d_step_rate(specs, steps: int = 5, warmup: int = 2, device: int = 0) -> dict:
    """The drop-in call surface used as the reference's driver uses it: one PM3D per peak,
    `a, delta = pm.step(a, da)` per step, each step returning the density grid to the host as
    float64 numpy (pbhgr/pbhgr/pm3d.py:117-129, pbhgr/scripts/pm3d_peak.py:26-28).  Wall clock
    per step, one peak per mesh size, weighted by the ensemble's composition."""
    import time

    from .pm3d import PM3D
    by_n = {}
    for s in specs:
        by_n.setdefault(s.N, []).append(s)
    total_ps, total_t, per = 0.0, 0.0, {}
    for N, group in sorted(by_n.items()):
        s = group[0]
        pm = PM3D(N, s.L, N, seed=s.seed, device=device).make_peak(s.R, s.delta0, s.noise_frac)
        a = 1.0
        for _ in range(warmup):
            a, _ = pm.step(a, a * s.ratio())
        t0 = time.perf_counter()
        for _ in range(steps):
            a, _ = pm.step(a, a * s.ratio())
        t_step = (time.perf_counter() - t0) / steps
        per[N] = t_step
        total_ps += len(group) * s.n
        total_t += len(group) * t_step
        pm.close()
    return {"particle_steps_per_s": total_ps / total_t, "step_s_by_mesh": {str(k): v for k, v in per.items()}}

