"""Served peak-collapse runs: a request loop with continuous batching on one GPU.

Each request is one recipe peak (pbh_b200.recipe.PeakSpec).  The server owns a pool of slots
(peaks of one engine in dynamic mode), a fixed number per mesh size, allocated once and sized
so that the pool's device memory stays inside the HBM budget.  At every engine step the loop

  1. admits queued requests whose size class has a free slot and whose footprint fits the
     budget still unused (initial conditions are generated on the device, noise included),
  2. advances every active slot by one step (one batched step for all of them: requests that
     arrived at different times run side by side, each on its own clock),
  3. retires runs that reached their collapse (first step with max delta >= delta_collapse) or
     their last step: the collapse time and the final density go back to the host and the
     slot is freed for the next request.

Latency is measured from a request's arrival to its result being on the host.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .engine import Engine, PeakConfig
from .ic import KIND_GAUSS, make_particles


@dataclass
class Request:
    rid: int
    spec: object                 # recipe.PeakSpec
    t_arrival: float             # seconds on the server clock
    t_admit: float = float("nan")
    t_done: float = float("nan")
    a_collapse_cfg: float = float("nan")   # -1: no collapse before the last step
    steps: int = 0
    delta: np.ndarray | None = None
    slot: int = -1

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


NATIVE_FFT_SIZES = (64, 128, 256, 512)   # meshes the engine transforms natively (no cuFFT work area)


def slot_bytes(N: int, native_fft: bool = True) -> int:
    """Device bytes one slot of mesh N holds in the engine (particles = cells)."""
    n = N ** 3
    per_particle = 2 * 16 + 2 * 16 + 2 * 4 + 2 * 4 + 4      # state x2, keys x2, values x2, bucket starts
    per_cell = 4 + 8 * (N // 2 + 1) / N * 4 + 12            # delta, 4 spectra, 3 force grids
    native = native_fft and N in NATIVE_FFT_SIZES
    fft_work = 0 if native else 16 * n                      # cuFFT's shared work area (~13-14 B per cell measured)
    return int(n * per_particle + n * per_cell + fft_work)


@dataclass
class ServerConfig:
    slots: dict = field(default_factory=lambda: {64: 32, 128: 32, 256: 32})
    tiles: object = None            # {N: super-tile side}, "auto" (autotuned) or None (default 16)
    budget_bytes: float = 150e9
    delta_collapse: float = 50.0
    keep_delta: bool = True
    device: int = 0


class Server:
    def __init__(self, cfg: ServerConfig):
        self.cfg = cfg
        torch = _lib.require_cuda()
        self._torch = torch
        tiles = cfg.tiles
        if tiles == "auto":
            from .tune import autotune
            tiles = autotune(cfg.slots, device=cfg.device)
        tiles = tiles or {}
        peaks, self.slot_N = [], []
        for N in sorted(cfg.slots):
            for _ in range(cfg.slots[N]):
                peaks.append(PeakConfig(N=N, Np=N, L=1.0, tile=int(tiles.get(N, 0))))
                self.slot_N.append(N)
        pool = sum(slot_bytes(N) for N in self.slot_N)
        if pool > cfg.budget_bytes:
            raise ValueError(f"slot pool needs {pool / 1e9:.1f} GB, over the {cfg.budget_bytes / 1e9:.0f} GB budget")
        self.engine = Engine(peaks, device=cfg.device, bucket_sort=True, graph=False, dynamic=True)
        self.free = {N: collections.deque(i for i, m in enumerate(self.slot_N) if m == N) for N in cfg.slots}
        self.active: dict[int, Request] = {}
        self.queue: collections.deque[Request] = collections.deque()
        self.done: list[Request] = []
        self.bytes_in_use = 0
        self.engine_steps = 0
        self.particle_steps = 0
        self._lib = _lib.load()

    # ---------------------------------------------------------------- requests
    def submit(self, req: Request):
        self.queue.append(req)

    def _admit(self, now: float):
        waiting = collections.deque()
        while self.queue:
            req = self.queue.popleft()
            N = req.spec.N
            fp = slot_bytes(N)
            if self.free.get(N) and self.bytes_in_use + fp <= self.cfg.budget_bytes:
                slot = self.free[N].popleft()
                s = req.spec
                x, p, _, _ = make_particles(N, N, s.L, KIND_GAUSS, s.delta0, s.R, noise_frac=s.noise_frac,
                                            device=self.cfg.device, noise_seed=s.seed + 1)
                self.engine.set_particles(slot, x, p, 1.0, mode=_lib.SCHED_RATIO, param=s.ratio(), max_steps=s.steps)
                self._lib.pm_set_collapse_threshold(self.engine._h, slot, float(self.cfg.delta_collapse), 1)
                del x, p
                req.slot, req.t_admit = slot, now
                self.active[slot] = req
                self.bytes_in_use += fp
            else:
                waiting.append(req)
        self.queue = waiting

    def _retire(self, now_fn):
        if not self.active:
            return
        clocks = (_lib.ClockInfo * self.engine.npeaks)()
        _lib.check(self._lib.pm_get_clocks_all(self.engine._h, clocks), "pm_get_clocks_all")
        for slot, req in list(self.active.items()):
            c = clocks[slot]
            if c.state == _lib.STATE_IDLE:
                req.steps = c.nsteps
                req.a_collapse_cfg = c.a_collapse / 100.0 if c.a_collapse > 0 else -1.0
                if self.cfg.keep_delta:
                    req.delta = self.engine.delta(slot).cpu().numpy()
                self.engine.release(slot)
                req.t_done = now_fn()
                self.free[req.spec.N].append(slot)
                self.free[req.spec.N] = collections.deque(sorted(self.free[req.spec.N]))
                self.bytes_in_use -= slot_bytes(req.spec.N)
                del self.active[slot]
                self.done.append(req)

    def step(self, now_fn):
        self._admit(now_fn())
        if not self.active:
            return False
        n_run = sum(r.spec.n for r in self.active.values())
        self.engine.run(1)
        self.engine_steps += 1
        self.particle_steps += n_run
        self._retire(now_fn)
        return True

    # ---------------------------------------------------------------- stream
    def serve(self, arrivals, timeout: float = 600.0):
        """Run a stream: `arrivals` is a list of (t_seconds, PeakSpec) in arrival order.
        Returns the completed requests.  Requests join the batch at the first step boundary
        after their arrival time."""
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        pending = collections.deque(Request(i, spec, t) for i, (t, spec) in enumerate(arrivals))
        total = len(pending)
        while len(self.done) < total and now() < timeout:
            while pending and pending[0].t_arrival <= now():
                self.submit(pending.popleft())
            busy = self.step(now)
            if not busy and not self.queue and pending:
                time.sleep(max(0.0, pending[0].t_arrival - now()))
        self.engine.sync()
        return self.done

    def close(self):
        self.engine.close()


def poisson_arrivals(rate: float, duration: float, seed: int = 7, sizes=(64, 128, 256), npeaks_max=None, steps=150):
    """Poisson arrivals of recipe peaks: mesh uniform over `sizes`, (e, p, delta0) as the
    batched ensemble (recipe.ensemble)."""
    from . import recipe
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (npeaks_max and len(out) >= npeaks_max):
            break
        spec = recipe.ensemble(npeaks=1, sizes=sizes, steps=steps, seed=int(rng.integers(1 << 30)))[0]
        out.append((t, spec))
    return out


def latency_summary(done) -> dict:
    lat = np.array([r.latency for r in done])
    if lat.size == 0:
        return {"completed": 0}
    return {"completed": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
