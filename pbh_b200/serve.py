"""Served peak-collapse runs: a request loop with continuous batching on one GPU.

Each request is one recipe peak (pbh_b200.recipe.PeakSpec).  The server owns a pool of slots
(peaks of one engine in dynamic mode), a fixed number per mesh size, allocated once and sized
so that the pool's device memory stays inside the HBM budget.  At every engine step the loop

  1. admits queued requests whose size class has a free slot and whose footprint fits the
     budget still unused: the initial particles are generated on a second stream (device noise
     included) and loaded into the slot on the engine's stream once they are ready,
  2. advances every active slot by one step (one batched step for all of them: requests that
     arrived at different times run side by side, each on its own clock),
  3. reads the clocks and statistics of the step before (a copy queued behind that step, so the
     host never waits for the step it has just queued) and retires runs that reached their
     collapse (first step with max delta >= delta_collapse) or their last step: the final
     density is copied to page-locked host memory behind the running work and the slot is
     freed for the next request.

The host therefore never waits on the device except for a step that is already followed by
another one in the queue.  Requests are refused at submission when they cannot run (a mesh
size without slots, a footprint over the budget, non-finite or non-positive parameters);
a run whose device status word turns nonzero (non-finite momentum, a lost particle, a sort
whose bounded wait gave up) ends as a failed request while the other slots keep stepping;
a request can be cancelled while queued or running.  The reference driver runs one peak per
process (pbhgr/scripts/pm3d_peak.py:20-34); the integer status convention follows
pbhgr/csrc/kernels.c:36,73.

Latency is measured from a request's arrival to its result being on the host.
"""
from __future__ import annotations

import collections
import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .engine import Engine, PeakConfig
from .ic import KIND_GAUSS


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
    ok: bool = True              # False: refused, cancelled or failed on the device (see error)
    error: str = ""
    status: int = 0              # the peak's device status word when it ended (pm_stats_info.status)
    admit_step: int = -1         # index of the engine step that primed it
    end_step: int = -1           # index of the engine step after which it was seen to have ended

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


NATIVE_FFT_SIZES = (64, 128, 256, 512)   # meshes the engine transforms natively (no cuFFT work area)


def slot_bytes(N: int, native_fft: bool = True) -> int:
    """Device bytes one slot of mesh N holds in the engine (particles = cells)."""
    n = N ** 3
    # two bin buffers with a quarter spare, the loading/overflow area, keys x2, values x2, tables
    per_particle = 2 * 32 * 5 / 4 + 32 + 2 * 4 + 2 * 4 + 4
    per_cell = 4 + 8 * (N // 2 + 1) / N * 4 + 12            # delta, 4 spectra, 3 force grids
    native = native_fft and N in NATIVE_FFT_SIZES
    fft_work = 0 if native else 16 * n                      # cuFFT's shared work area (~13-14 B per cell measured)
    return int(n * per_particle + n * per_cell + fft_work)


def ic_buffer_bytes(N: int) -> int:
    """Device bytes of one initial-condition buffer (float64 positions and momenta)."""
    return 2 * 3 * 8 * N ** 3


@dataclass
class ServerConfig:
    slots: dict = field(default_factory=lambda: {64: 32, 128: 32, 256: 32})
    tiles: object = None            # {N: super-tile side}, "auto" (autotuned) or None (default 16)
    budget_bytes: float = 150e9
    delta_collapse: float = 50.0
    keep_delta: bool = True
    device: int = 0
    ic_buffers: int = 2             # initial-condition buffers per mesh size (admissions per step)


def refusal_reason(spec, cfg: ServerConfig) -> str:
    """Why a request cannot run on a server of this configuration ("" if it can): a mesh size
    without slots, a slot footprint over the budget, non-finite or non-positive parameters."""
    N = getattr(spec, "N", None)
    if N not in cfg.slots or cfg.slots[N] < 1:
        return f"refused: no slots of mesh {N}"
    if slot_bytes(N) + cfg.ic_buffers * ic_buffer_bytes(N) > cfg.budget_bytes:
        return "refused: footprint over the HBM budget"
    try:
        vals = [float(v) for v in (spec.delta0, spec.e, spec.p, spec.L, spec.noise_frac, *spec.R)]
    except (TypeError, ValueError):
        return "refused: non-numeric parameter"
    if not all(math.isfinite(v) for v in vals):
        return "refused: non-finite parameter"
    if spec.delta0 <= 0 or min(spec.R) <= 0 or spec.L <= 0 or spec.noise_frac < 0 or int(spec.steps) < 1:
        return "refused: delta0, R, L and steps must be positive"
    return ""


class _ICBuffer:
    """Float64 particle buffers an admission's initial conditions are generated into; free
    again once the engine's stream has loaded them (event `loaded`)."""

    def __init__(self, torch, N: int, device: int):
        n = N ** 3
        self.x = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{device}")
        self.p = torch.empty_like(self.x)
        self.loaded = None

    def ready(self) -> bool:
        return self.loaded is None or self.loaded.query()


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
        pool = sum(slot_bytes(N) for N in self.slot_N) + sum(cfg.ic_buffers * ic_buffer_bytes(N) for N in cfg.slots)
        if pool > cfg.budget_bytes:
            raise ValueError(f"slot pool needs {pool / 1e9:.1f} GB, over the {cfg.budget_bytes / 1e9:.0f} GB budget")
        self.engine = Engine(peaks, device=cfg.device, bucket_sort=True, graph=False, dynamic=True)
        self._h = self.engine._h
        self._lib = _lib.load()
        dev = f"cuda:{cfg.device}"
        self._estream = torch.cuda.ExternalStream(self._lib.pm_engine_stream(self._h), device=dev)
        self._icstream = torch.cuda.Stream(device=dev)
        self._icbuf = {N: [_ICBuffer(torch, N, cfg.device) for _ in range(cfg.ic_buffers)] for N in cfg.slots}
        self._pinned = {N: [] for N in cfg.slots}      # page-locked delta buffers, reused
        self.free = {N: collections.deque(i for i, m in enumerate(self.slot_N) if m == N) for N in cfg.slots}
        self.active: dict[int, Request] = {}
        self.queue: collections.deque[Request] = collections.deque()
        self.done: list[Request] = []
        self._finishing: list = []                     # (request, event, pinned buffer)
        self._pending = collections.deque()            # snapshot step indices not read yet
        self._clocks = (_lib.ClockInfo * len(peaks))()
        self._stats = (_lib.StatsInfo * len(peaks))()
        self.bytes_in_use = 0
        self.engine_steps = 0
        self.particle_steps = 0
        self.step_wall = []                            # host seconds per loop iteration with a step
        self._t0 = time.perf_counter()

    # ---------------------------------------------------------------- requests
    def _refusal(self, spec) -> str:
        return refusal_reason(spec, self.cfg)

    def _finish(self, req: Request, t: float, ok: bool = True, error: str = ""):
        req.t_done = t
        req.ok = ok
        req.error = error
        self.done.append(req)

    def submit(self, req: Request, now: float | None = None):
        why = self._refusal(req.spec)
        if why:
            self._finish(req, req.t_arrival if now is None else now, ok=False, error=why)
        else:
            self.queue.append(req)

    def cancel(self, rid: int, now: float) -> bool:
        """End a queued or running request; returns False if it is not queued or running."""
        for req in list(self.queue):
            if req.rid == rid:
                self.queue.remove(req)
                self._finish(req, now, ok=False, error="cancelled")
                return True
        for slot, req in list(self.active.items()):
            if req.rid == rid:
                self._free_slot(slot)
                self._finish(req, now, ok=False, error="cancelled")
                return True
        return False

    def _free_slot(self, slot: int):
        req = self.active.pop(slot)
        _lib.check(self._lib.pm_release(self._h, slot), "pm_release")
        self.free[req.spec.N].append(slot)
        self.free[req.spec.N] = collections.deque(sorted(self.free[req.spec.N]))
        self.bytes_in_use -= slot_bytes(req.spec.N)

    def _admit(self, now: float):
        waiting = collections.deque()
        torch = self._torch
        while self.queue:
            req = self.queue.popleft()
            N = req.spec.N
            fp = slot_bytes(N)
            buf = next((b for b in self._icbuf[N] if b.ready()), None)
            if not (self.free[N] and self.bytes_in_use + fp <= self.cfg.budget_bytes and buf is not None):
                waiting.append(req)
                continue
            slot = self.free[N].popleft()
            s = req.spec
            prm = _lib.ICParams()
            prm.N, prm.Np, prm.L, prm.kind, prm.amp = N, N, float(s.L), KIND_GAUSS, float(s.delta0)
            prm.axes = (ctypes.c_double * 3)(*[float(v) for v in s.R])
            prm.noise_frac = float(s.noise_frac)
            prm.noise_seed = int(s.seed) + 1
            # the buffer's previous load has finished (ready()), so the IC stream may overwrite it
            _lib.check(self._lib.pm_make_ic_async(ctypes.byref(prm), buf.x.data_ptr(), buf.p.data_ptr(),
                                                  self._icstream.cuda_stream), "pm_make_ic_async")
            made = torch.cuda.Event()
            made.record(self._icstream)
            _lib.check(self._lib.pm_load_peak(self._h, slot, buf.x.data_ptr(), buf.p.data_ptr(), 1.0,
                                              _lib.SCHED_RATIO, float(s.ratio()), 0.0, int(s.steps),
                                              float(self.cfg.delta_collapse), 1, made.cuda_event), "pm_load_peak")
            buf.loaded = torch.cuda.Event()
            buf.loaded.record(self._estream)
            req.slot, req.t_admit, req.admit_step = slot, now, self.engine_steps
            self.active[slot] = req
            self.bytes_in_use += fp
        self.queue = waiting

    def _read_snapshot(self, step_index: int):
        """Retire from the clocks and statistics copied after engine step `step_index`."""
        _lib.check(self._lib.pm_snapshot_read(self._h, step_index % 2, 1, self._clocks, self._stats),
                   "pm_snapshot_read")
        for slot, req in list(self.active.items()):
            if req.admit_step > step_index:          # loaded after this snapshot was taken
                continue
            c, st = self._clocks[slot], self._stats[slot]
            if st.status:
                req.status = int(st.status)
                req.steps = c.nsteps
                req.end_step = step_index
                self._free_slot(slot)
                self._finish(req, time.perf_counter() - self._t0, ok=False,
                             error=f"device status 0x{req.status:x}")
                continue
            if c.state != _lib.STATE_IDLE:
                continue
            req.steps = c.nsteps
            req.end_step = step_index
            req.a_collapse_cfg = c.a_collapse / 100.0 if c.a_collapse > 0 else -1.0
            pinned = None
            if self.cfg.keep_delta:
                pool = self._pinned[req.spec.N]
                pinned = pool.pop() if pool else self._torch.empty(req.spec.N ** 3, dtype=self._torch.float32,
                                                                   pin_memory=True)
                _lib.check(self._lib.pm_get_delta_async(self._h, slot, pinned.data_ptr()), "pm_get_delta_async")
            self._free_slot(slot)
            ev = self._torch.cuda.Event()
            ev.record(self._estream)
            self._finishing.append((req, ev, pinned))

    def _collect(self, now_fn, wait: bool = False):
        keep = []
        for req, ev, pinned in self._finishing:
            if wait:
                ev.synchronize()
            if ev.query():
                if pinned is not None:
                    N = req.spec.N
                    req.delta = pinned.numpy().reshape(N, N, N).copy()
                    self._pinned[N].append(pinned)
                self._finish(req, now_fn())
            else:
                keep.append((req, ev, pinned))
        self._finishing = keep

    def step(self, now_fn) -> bool:
        """One iteration of the loop: admit, queue one engine step, retire from the step before.
        Returns False when there was nothing to do."""
        t_it = time.perf_counter()
        self._admit(now_fn())
        if self.active:
            n_run = sum(r.spec.n for r in self.active.values())
            if len(self._pending) == 2:               # both snapshot buffers hold unread copies
                self._read_snapshot(self._pending.popleft())
            _lib.check(self._lib.pm_run(self._h, 1), "pm_run")
            _lib.check(self._lib.pm_snapshot(self._h, self.engine_steps % 2), "pm_snapshot")
            self._pending.append(self.engine_steps)
            self.engine_steps += 1
            self.particle_steps += n_run
            if len(self._pending) == 2:               # the step before, while this one is queued
                self._read_snapshot(self._pending.popleft())
            self._collect(now_fn)
            self.step_wall.append(time.perf_counter() - t_it)
            return True
        busy = bool(self._pending or self._finishing)
        while self._pending:
            self._read_snapshot(self._pending.popleft())
        self._collect(now_fn, wait=not self.active and not self.queue)
        return busy

    # ---------------------------------------------------------------- stream
    def serve(self, arrivals, timeout: float = 600.0, cancel_at=None):
        """Run a stream: `arrivals` is a list of (t_seconds, PeakSpec) in arrival order.
        Returns the ended requests (completed, refused, cancelled or failed; Request.ok tells).
        Requests join the batch at the first step boundary after their arrival time.
        cancel_at: optional {request index: seconds} of cancellations."""
        self._t0 = t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        pending = collections.deque(Request(i, spec, t) for i, (t, spec) in enumerate(arrivals))
        cancels = sorted((t, rid) for rid, t in (cancel_at or {}).items())
        total = len(pending)
        while len(self.done) < total and now() < timeout:
            while pending and pending[0].t_arrival <= now():
                self.submit(pending.popleft(), now())
            while cancels and cancels[0][0] <= now():
                self.cancel(cancels.pop(0)[1], now())
            busy = self.step(now)
            if not busy and not self.queue and pending:
                time.sleep(max(0.0, pending[0].t_arrival - now()))
        self.engine.sync()
        self._collect(now, wait=True)
        return self.done

    def close(self):
        self.engine.sync()
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
    ok = [r for r in done if r.ok]
    lat = np.array([r.latency for r in ok])
    out = {"completed": int(lat.size), "failed": int(len(done) - len(ok))}
    if lat.size:
        out.update(p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                   mean_s=float(lat.mean()), max_s=float(lat.max()))
    return out
