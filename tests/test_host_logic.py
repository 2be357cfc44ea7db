"""Host-side logic that needs no GPU: the benchmark recipes, the served stream's arrivals,
latency summary, slot budget and retire/fail/cancel decisions (the device replaced by a script),
the benchmark's launch and byte accounting, its CPU sample and reference-arm line, and the error
mapping of the C ABI's return codes."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def test_zeldovich_axes_and_implied_ep_invert_each_other():
    from pbh_b200 import recipe
    for e, p in [(0.0, 0.0), (0.2, 0.0), (0.3, 0.1), (0.1, -0.05)]:
        A = recipe.zeldovich_axes(e, p)
        assert np.prod(A) == pytest.approx(1.0, rel=1e-12)
        lam = np.array([1 + 3 * e + p, 1 - 2 * p, 1 - 3 * e + p]) / 3.0     # pm3d.py:20-23
        assert A == pytest.approx(lam ** -0.5 / np.prod(lam ** -0.5) ** (1 / 3), rel=1e-12)
        e2, p2 = recipe.implied_ep(A)
        assert (e2, p2) == pytest.approx((e, p), abs=1e-12)


def test_step_ratio_spans_a_factor_100():
    from pbh_b200 import recipe
    for steps in (50, 100, 150, 300):
        spec = recipe.single_peak(N=32, steps=steps)
        assert (1.0 + spec.ratio()) ** steps == pytest.approx(100.0, rel=1e-12)


def test_spherical_delta0_is_the_linear_threshold():
    from pbh_b200 import recipe
    # e = p = 0: the first axis collapses with the sphere, delta_lin(a_c) = 1.686
    assert recipe.first_axis_ratio(0.0, 0.0) == pytest.approx(1.0)
    for a_c in (0.3, 0.5, 0.8, 1.0):
        d0 = recipe.delta0_for_collapse(a_c, 0.0, 0.0)
        assert d0 * a_c / recipe.A_START_CFG == pytest.approx(recipe.DELTA_C, rel=1e-12)
    # an ellipsoid's first axis collapses earlier, so it needs less initial overdensity
    assert recipe.delta0_for_collapse(0.8, 0.3, 0.1) < recipe.delta0_for_collapse(0.8, 0.0, 0.0)


def test_ensemble_is_seeded_and_within_its_ranges():
    from pbh_b200 import recipe
    a = recipe.ensemble(npeaks=64, seed=1234)
    b = recipe.ensemble(npeaks=64, seed=1234)
    assert [(s.N, s.e, s.p, s.delta0, s.seed) for s in a] == [(s.N, s.e, s.p, s.delta0, s.seed) for s in b]
    assert {s.N for s in a} <= {32, 64, 128, 256}
    assert all(0.0 <= s.e <= 0.3 and -0.1 <= s.p <= 0.1 and 0.3 <= s.a_collapse_cfg <= 1.0 for s in a)
    assert [s.seed for s in a] == list(range(1234, 1234 + 64))
    assert sum(s.n for s in a) >= 1e8


def test_poisson_arrivals_are_seeded_and_ordered():
    from pbh_b200.serve import poisson_arrivals
    a = poisson_arrivals(rate=20.0, duration=10.0, seed=3)
    b = poisson_arrivals(rate=20.0, duration=10.0, seed=3)
    assert [(t, s.N, s.seed) for t, s in a] == [(t, s.N, s.seed) for t, s in b]
    times = [t for t, _ in a]
    assert times == sorted(times) and 0.0 < times[0] and times[-1] <= 10.0
    assert 120 <= len(a) <= 280                      # 200 expected
    assert {s.N for _, s in a} <= {64, 128, 256}
    assert len(poisson_arrivals(rate=20.0, duration=10.0, seed=3, npeaks_max=5)) == 5


def test_latency_summary():
    from pbh_b200.serve import Request, latency_summary
    done = []
    for i, lat in enumerate(np.linspace(1.0, 2.0, 101)):
        r = Request(rid=i, spec=None, t_arrival=10.0)
        r.t_done = 10.0 + lat
        done.append(r)
    s = latency_summary(done)
    assert s["completed"] == 101
    assert s["p50_s"] == pytest.approx(1.5) and s["max_s"] == pytest.approx(2.0)
    assert s["p99_s"] == pytest.approx(1.99)
    assert s["failed"] == 0
    assert latency_summary([]) == {"completed": 0, "failed": 0}
    # refused, cancelled and failed requests are counted apart, not in the latencies
    bad = Request(rid=999, spec=None, t_arrival=0.0, ok=False, error="cancelled")
    bad.t_done = 1e6
    s2 = latency_summary(done + [bad])
    assert s2["completed"] == 101 and s2["failed"] == 1 and s2["max_s"] == pytest.approx(2.0)


def test_served_slot_pool_fits_the_budget():
    from pbh_b200.serve import slot_bytes
    sizes = [slot_bytes(n) for n in (64, 128, 256)]
    assert sizes == sorted(sizes)
    # per particle the same, less the cuFFT work area that the native transform does not use
    assert slot_bytes(256) == pytest.approx(8 * slot_bytes(128), rel=0.01)
    assert slot_bytes(256) == slot_bytes(256, native_fft=False) - 16 * 256 ** 3
    assert slot_bytes(32) == slot_bytes(32, native_fft=False)            # cuFFT at 32^3 either way
    pool = 32 * slot_bytes(64) + 32 * slot_bytes(128) + 24 * slot_bytes(256)  # the served benchmark's pool
    assert pool <= 150e9


def test_engine_flags():
    """The engine flags word: no super-tile re-sort by default, a period when asked for, every
    step without bucketed regrouping; the feature bits."""
    from pbh_b200 import _lib
    from pbh_b200.engine import engine_flags
    period = lambda f: (f >> 8) & 0xFF
    assert period(engine_flags()) == 0
    assert period(engine_flags(full_every=16)) == 16
    assert period(engine_flags(full_every=1000)) == 255
    assert period(engine_flags(full_every=16, bucket_sort=False)) == 1
    f = engine_flags(graph=False, dynamic=True, native_fft=False, tight_bins=True)
    assert not f & _lib.FLAG_GRAPH and f & _lib.FLAG_DYNAMIC and not f & _lib.FLAG_NATIVE_FFT
    assert f & _lib.FLAG_TIGHT_BINS
    assert engine_flags() & _lib.FLAG_GRAPH and engine_flags() & _lib.FLAG_NATIVE_FFT


def test_launch_accounting():
    import bench
    assert bench.launches_per_step([32], "native") == 10              # cuFFT size only
    assert bench.launches_per_step([32, 64], "native") == 16          # 64^3 native, Green for 32^3
    assert bench.launches_per_step([32, 64, 128, 256], "native") == 28  # the batched ensemble
    assert bench.launches_per_step([256], "cufft") == 10
    assert bench.launches_per_step([256], "native") == 15             # + 6, no Green launch
    assert bench.launches_per_step([512], "native") == 15
    assert bench.launches_per_step([32, 256, 256], "native") == 16    # Green still runs for 32^3
    assert bench.launches_per_step([256, 512], "native") == 21


def test_algorithmic_bytes_per_phase():
    import bench
    n, cells, modes = 1000, 1000, 600
    assert bench.algorithmic_bytes("push", n, cells, modes, 3) == n * 64 + cells * 12
    assert bench.algorithmic_bytes("refresh", n, cells, modes, 3) == n * 64
    assert bench.algorithmic_bytes("regroup", n, cells, modes, 3) == 0.0   # relayouts only on overflow
    assert bench.algorithmic_bytes("deposit", n, cells, modes, 3) == n * 16 + cells * 4
    assert bench.algorithmic_bytes("green", n, cells, modes, 3) == modes * 32
    assert bench.algorithmic_bytes("r2c", n, cells, modes, 3) == 0.0


def test_cpu_sample_covers_every_mesh_size_of_the_mix():
    """The CPU baseline samples every mesh size of the workload, loads the cores roughly in
    proportion to each size's particles, stays inside the host memory it is given, and turns
    per-size per-core rates into the rate of the whole mix."""
    import bench
    specs, _ = bench.workload_specs("batched", 64, 1234, 0)
    pm = {}
    for s in specs:
        pm[s.N] = pm.get(s.N, 0) + s.n
    assert sorted(pm) == [32, 64, 128, 256]
    alloc = bench.allocate_cpu_workers(pm, 16, 1e12)
    assert sorted(alloc) == [32, 64, 128, 256] and sum(alloc.values()) == 16
    assert alloc[256] == max(alloc.values())                     # most of the mix's particles
    need = lambda a: sum(k * (bench.CPU_BYTES_PER_PARTICLE * N ** 3 + bench.CPU_BYTES_PER_WORKER)
                         for N, k in a.items())
    tight = bench.allocate_cpu_workers(pm, 16, 20e9)
    assert need(tight) <= 20e9 and tight[256] >= 1 and sum(tight.values()) <= 16
    assert bench.allocate_cpu_workers(pm, 2, 1e12) == {256: 1, 128: 1}   # fewer cores than sizes
    assert 256 not in bench.allocate_cpu_workers(pm, 16, 5e9)    # one 256^3 peak does not fit
    # Equal per-core rates: the mix runs at cores x that rate; a slower size weighs by its particles.
    assert bench.mix_rate(pm, {N: 1e6 for N in pm}, 16) == pytest.approx(16e6)
    r = {32: 2e6, 64: 2e6, 128: 2e6, 256: 1e6}
    p_tot = sum(pm.values())
    expect = 16 * p_tot / (pm[256] / 1e6 + (p_tot - pm[256]) / 2e6)
    assert bench.mix_rate(pm, r, 16) == pytest.approx(expect)


def test_cpu_sample_runs_and_survives_a_failing_worker():
    """The CPU sample end to end on small meshes (spawned workers, a common timed window), and a
    worker that fails before the window (a negative seed, which numpy's generator rejects): it is
    reported, and the others are still timed and give the mix's rate."""
    import dataclasses

    import bench
    from pbh_b200 import recipe
    specs = recipe.ensemble(npeaks=6, sizes=(8, 16), steps=100, seed=5)
    cb = bench.cpu_rate(specs, budget=0.3, warmup=1, workers=3)
    assert cb["cores"] == 3 and cb["errors"] is None and cb["value"] > 0
    assert sorted(cb["per_core_rate_by_mesh"]) == sorted(str(N) for N in {s.N for s in specs})
    bad = [dataclasses.replace(s, seed=-1) if s.N == 16 else s for s in specs]
    cb = bench.cpu_rate(bad, budget=0.3, warmup=1, workers=3)
    assert cb["errors"] and all("16^3" in e for e in cb["errors"])
    assert cb["cores"] == 3 - len(cb["errors"]) and cb["value"] > 0
    assert list(cb["per_core_rate_by_mesh"]) == ["8"]        # 16^3 takes the measured size's rate


def test_return_code_mapping():
    from pbh_b200 import _lib
    assert _lib.check(0, "x") == 0 and _lib.check(3, "x") == 3        # >0: flagged items
    with pytest.raises(_lib.PMError, match="CUDA error 2"):
        _lib.check(-2, "x")
    with pytest.raises(_lib.PMError, match="cuFFT error 5"):
        _lib.check(-1005, "x")
    with pytest.raises(_lib.PMError, match="invalid argument"):
        _lib.check(-2003, "x")


def test_served_requests_are_refused_for_the_right_reasons():
    import dataclasses

    from pbh_b200 import recipe
    from pbh_b200.serve import ServerConfig, refusal_reason
    cfg = ServerConfig(slots={64: 2, 128: 1}, budget_bytes=150e9)
    ok = recipe.ensemble(npeaks=1, sizes=(64,), seed=3)[0]
    assert refusal_reason(ok, cfg) == ""
    cases = {"no slots": dataclasses.replace(ok, N=256),
             "non-finite": dataclasses.replace(ok, delta0=float("nan")),
             "positive": dataclasses.replace(ok, delta0=-0.01)}
    for why, spec in cases.items():
        assert why in refusal_reason(spec, cfg), why
    assert "positive" in refusal_reason(dataclasses.replace(ok, R=(0.1, 0.0, 0.1)), cfg)
    assert "positive" in refusal_reason(dataclasses.replace(ok, steps=0), cfg)
    tiny = ServerConfig(slots={64: 1}, budget_bytes=1e6)
    assert "budget" in refusal_reason(ok, tiny)


def test_state_arrays_track_writes_like_the_references_plain_arrays():
    """PM3D.x / PM3D.p are host copies of device state: writing into them (items, slices,
    in-place arithmetic, ufunc out=, through views) must mark them for loading back, and a copy
    from before the device state changed must not."""
    from types import SimpleNamespace

    from pbh_b200.pm3d import StateArray
    owner = SimpleNamespace(_host_gen=3, _host_dirty=False)

    def fresh(gen=3):
        a = np.zeros((10, 3)).view(StateArray)
        a._owner, a._gen = owner, gen
        owner._host_dirty = False
        return a

    a = fresh()
    a[2] = 1.0
    assert owner._host_dirty and a[2, 1] == 1.0
    a = fresh()
    a[:, 0] *= 2.0                                   # __setitem__ of the augmented assignment
    assert owner._host_dirty
    a = fresh()
    np.add(a, 1.0, out=a)
    assert owner._host_dirty and np.all(a == 1.0)
    a = fresh()
    v = a[3:5]
    v[0, 0] = 7.0                                    # a view writes through and marks the owner
    assert owner._host_dirty and a[3, 0] == 7.0
    a = fresh()
    b = a + 1.0                                      # a new array is not the state
    assert not owner._host_dirty and isinstance(b, np.ndarray)
    s = fresh(gen=2)                                 # stale copy from an earlier state
    s[0] = 5.0
    assert not owner._host_dirty
    a = fresh()
    c = a.copy()                                     # a copy is a snapshot, not the state
    c[0] = 9.0
    assert not owner._host_dirty and a[0, 0] == 0.0


def test_reference_arm_prints_one_contract_line(monkeypatch, capsys):
    """`bench.py --impl reference` prints one JSON line with the contract's keys, the workload's
    own config and a cpu_baseline describing the sample (small meshes stand in for the mix)."""
    import argparse
    import json

    import bench
    from pbh_b200 import recipe
    small = recipe.ensemble(npeaks=4, sizes=(8, 16), steps=100, seed=3)
    monkeypatch.setattr(bench, "workload_specs", lambda name, npeaks, seed, rank: (small, {"workload": "small mix"}))
    monkeypatch.delenv("RANK", raising=False)
    args = argparse.Namespace(workload="batched", npeaks=4, seed=1, gpus=1, steps=20, warmup=5, cpu_seconds=0.2)
    bench.run_reference(args)
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["value"] > 0 and (d["steps"], d["warmup"]) == (20, 5)
    assert d["config"]["workload"] == "small mix" and d["config"]["peaks"] == 4
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    monkeypatch.setenv("RANK", "1")                      # other ranks of a multi-GPU launch print nothing
    bench.run_reference(args)
    assert capsys.readouterr().out.strip() == ""


class _FakeEvent:
    def record(self, stream=None):
        pass

    def query(self):
        return True

    def synchronize(self):
        pass


class _FakeTorch:
    """The few torch calls the served loop's retire path makes, on the CPU."""
    float32 = None

    class cuda:
        Event = _FakeEvent

    @staticmethod
    def empty(n, dtype=None, pin_memory=False):
        import torch
        return torch.zeros(n, dtype=torch.float32)


class _FakeServedLib:
    """Stands in for libpmb200's served-loop entry points: pm_snapshot_read fills the clocks and
    statistics from a script, pm_release and pm_get_delta_async record their calls."""

    def __init__(self, script):
        self.script, self.released, self.delta_copies = script, [], []

    def pm_snapshot_read(self, h, slot, wait, clocks, stats):
        for peak, (state, nsteps, a_collapse, status) in self.script.items():
            clocks[peak].state, clocks[peak].nsteps, clocks[peak].a_collapse = state, nsteps, a_collapse
            stats[peak].status = status
        return 0

    def pm_release(self, h, peak):
        self.released.append(peak)
        return 0

    def pm_get_delta_async(self, h, peak, dst):
        self.delta_copies.append(peak)
        return 0


def _server_on_fakes(script, nslots=3, N=8):
    """A Server whose engine is replaced by `_FakeServedLib` (its host-side bookkeeping only)."""
    import collections
    import time

    from pbh_b200 import _lib
    from pbh_b200.serve import Server, ServerConfig
    srv = Server.__new__(Server)
    srv.cfg = ServerConfig(slots={N: nslots}, keep_delta=True)
    srv._lib, srv._h, srv._torch, srv._estream = _FakeServedLib(script), None, _FakeTorch, None
    srv.slot_N = [N] * nslots
    srv.free = {N: collections.deque()}          # every slot busy
    srv.active, srv.queue, srv.done = {}, collections.deque(), []
    srv._finishing, srv._pending, srv._pinned = [], collections.deque(), {N: []}
    srv._clocks = (_lib.ClockInfo * nslots)()
    srv._stats = (_lib.StatsInfo * nslots)()
    srv.bytes_in_use, srv.engine_steps, srv._t0 = 0, 5, time.perf_counter()
    return srv


def test_served_loop_retires_fails_and_cancels_runs_on_the_host():
    """The served loop's decisions from a step's snapshot, with the device replaced by a script:
    a peak whose clock went idle completes (collapse a in the config's units, its delta copied
    out behind the running work), a peak whose status word is nonzero fails while the others go
    on, a run loaded after the snapshot was taken is not judged by it, and cancelling frees a
    running slot or drops a queued request.  Every freed slot returns to the pool."""
    from pbh_b200 import _lib, recipe
    from pbh_b200.serve import Request, slot_bytes
    N = 8
    script = {0: (_lib.STATE_IDLE, 40, 55.0, 0),      # collapsed at a_pm = 55 -> a_cfg = 0.55
              1: (_lib.STATE_RUN, 12, -1.0, 0x1),     # non-finite momentum
              2: (_lib.STATE_IDLE, 0, -1.0, 0)}       # loaded after the snapshot: not judged yet
    srv = _server_on_fakes(script, N=N)
    spec = recipe.ensemble(npeaks=1, sizes=(N,), seed=2)[0]
    reqs = [Request(rid=i, spec=spec, t_arrival=0.0) for i in range(4)]
    for slot, admit in ((0, 3), (1, 3), (2, 6)):
        reqs[slot].slot, reqs[slot].admit_step = slot, admit
        srv.active[slot] = reqs[slot]
        srv.bytes_in_use += slot_bytes(N)
    srv.queue.append(reqs[3])
    srv._read_snapshot(4)
    assert srv._lib.released == [0, 1] and srv._lib.delta_copies == [0]
    failed = [r for r in srv.done if not r.ok]
    assert [r.rid for r in failed] == [1] and failed[0].status == 1 and "0x1" in failed[0].error
    assert list(srv.active) == [2] and [r.rid for r, _, _ in srv._finishing] == [0]
    srv._collect(lambda: 1.0)
    done0 = next(r for r in srv.done if r.rid == 0)
    assert done0.ok and done0.steps == 40 and done0.a_collapse_cfg == pytest.approx(0.55)
    assert done0.delta.shape == (N, N, N) and done0.t_done == 1.0
    assert srv.cancel(2, now=2.0) and srv.cancel(3, now=2.0) and not srv.cancel(99, now=2.0)
    assert srv._lib.released == [0, 1, 2] and not srv.active and not srv.queue
    assert {r.rid: r.error for r in srv.done if not r.ok} == {1: "device status 0x1", 2: "cancelled",
                                                            3: "cancelled"}
    assert sorted(srv.free[N]) == [0, 1, 2] and srv.bytes_in_use == 0


def test_served_admission_waits_for_a_slot_an_ic_buffer_and_budget():
    """Admission on the host, the device replaced by recorders: a queued request starts only when
    its mesh size has a free slot, an initial-condition buffer whose last load has finished, and
    room under the HBM budget; the others keep their order in the queue."""
    import collections

    from pbh_b200 import recipe
    from pbh_b200.serve import Request, slot_bytes
    N = 8

    class Ev(_FakeEvent):
        done = False                                   # the engine's stream has passed every load
        cuda_event = None

        def query(self):
            return Ev.done

    class Buf:                                         # serve._ICBuffer with host stand-ins
        def __init__(self, loaded):
            self.loaded = loaded
            self.x = self.p = type("T", (), {"data_ptr": lambda self: 0})()

        def ready(self):
            return self.loaded is None or self.loaded.query()

    calls = []

    class Lib(_FakeServedLib):
        def pm_make_ic_async(self, prm, x, p, stream):
            prm = prm._obj                              # ctypes.byref(ICParams)
            calls.append(("ic", prm.N, prm.noise_seed))
            return 0

        def pm_load_peak(self, h, slot, *args):
            calls.append(("load", slot))
            return 0

    srv = _server_on_fakes({}, nslots=3, N=N)
    srv._lib = Lib({})
    srv._torch = type("FT", (), {"cuda": type("C", (), {"Event": Ev})})
    srv._icstream = type("S", (), {"cuda_stream": None})()
    srv.free = {N: collections.deque([0, 1, 2])}
    srv._icbuf = {N: [Buf(None), Buf(Ev())]}           # one buffer free, one still loading
    spec = recipe.ensemble(npeaks=1, sizes=(N,), seed=2)[0]
    for i in range(3):
        srv.queue.append(Request(rid=i, spec=spec, t_arrival=0.0))
    srv._admit(0.0)
    assert list(srv.active) == [0] and [r.rid for r in srv.queue] == [1, 2]
    assert calls == [("ic", N, spec.seed + 1), ("load", 0)] and srv.bytes_in_use == slot_bytes(N)
    # the loads have finished, so both buffers are free again, but the budget holds one more slot
    Ev.done = True
    srv.cfg.budget_bytes = 2 * slot_bytes(N)
    srv._admit(1.0)
    assert sorted(srv.active) == [0, 1] and [r.rid for r in srv.queue] == [2]
    srv._admit(2.0)                                    # buffers free, slot free, budget full
    assert sorted(srv.active) == [0, 1] and [r.rid for r in srv.queue] == [2]
    srv.cfg.budget_bytes = 150e9
    srv._admit(3.0)
    assert sorted(srv.active) == [0, 1, 2] and not srv.queue and srv.active[2].admit_step == srv.engine_steps
