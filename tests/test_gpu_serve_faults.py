"""Failure handling of the served loop, with no GPU fault: bad requests are refused at the door,
cancelled requests end without a result, a run whose device status word turns nonzero ends as
a failed request while the others complete, and a bounded wait of the sort that runs out (on
look-back words that nothing publishes) reaches the caller as a status, not a hang."""
import dataclasses
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def specs(n, sizes=(16, 32), steps=30, seed=5):
    from pbh_b200 import recipe
    return recipe.ensemble(npeaks=n, sizes=sizes, steps=steps, seed=seed, a_range=(0.02, 0.05))


def test_bad_requests_are_refused_and_the_rest_complete():
    from pbh_b200.serve import Server, ServerConfig
    good = specs(3)
    bad = [dataclasses.replace(good[0], delta0=float("nan")),          # non-finite
           dataclasses.replace(good[1], delta0=-0.05),                  # a void: no collapse to detect
           dataclasses.replace(good[2], N=512),                         # no slot class holds it
           dataclasses.replace(good[0], R=(0.1, 0.0, 0.1))]             # degenerate axis
    srv = Server(ServerConfig(slots={16: 2, 32: 2}, budget_bytes=20e9, delta_collapse=2.0))
    arrivals = [(0.0, s) for s in good[:2]] + [(0.01, s) for s in bad] + [(0.02, good[2])]
    done = {r.rid: r for r in srv.serve(arrivals)}
    srv.close()
    assert len(done) == len(arrivals)
    for rid in range(2, 2 + len(bad)):
        assert not done[rid].ok and done[rid].error.startswith("refused"), done[rid]
        assert done[rid].delta is None
    for rid in (0, 1, len(arrivals) - 1):
        r = done[rid]
        assert r.ok and r.status == 0 and r.delta is not None and r.steps > 0, r


def test_cancelled_requests_end_and_others_keep_stepping():
    from pbh_b200.serve import Request, Server, ServerConfig
    sp = specs(4, sizes=(32,), steps=60)
    srv = Server(ServerConfig(slots={32: 2}, budget_bytes=20e9, delta_collapse=0.0))   # no early stop
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for i, s in enumerate(sp):
        srv.submit(Request(i, s, 0.0), now())
    for _ in range(5):
        srv.step(now)
    # requests 0 and 1 run in the two slots; 2 and 3 wait for a slot
    assert sorted(r.rid for r in srv.active.values()) == [0, 1]
    assert srv.cancel(0, now())                       # running
    assert srv.cancel(3, now())                       # still queued
    assert not srv.cancel(3, now())
    while len(srv.done) < 4:
        srv.step(now)
    srv.close()
    done = {r.rid: r for r in srv.done}
    assert not done[0].ok and done[0].error == "cancelled"
    assert not done[3].ok and done[3].error == "cancelled" and np.isnan(done[3].t_admit)
    for rid in (1, 2):
        assert done[rid].ok and done[rid].steps == 60, done[rid]


def test_non_finite_run_fails_alone():
    """A peak whose momenta overflow FP32 (an absurd amplitude) raises status bit 0 on the device:
    that request fails, the one beside it completes with the same result as alone."""
    from pbh_b200.serve import Server, ServerConfig
    sp = specs(2, sizes=(32,), steps=20)
    blow = dataclasses.replace(sp[0], delta0=1e300)
    cfg = ServerConfig(slots={32: 2}, budget_bytes=20e9, delta_collapse=0.0)
    srv = Server(cfg)
    done = {r.rid: r for r in srv.serve([(0.0, blow), (0.0, sp[1])])}
    srv.close()
    assert not done[0].ok and done[0].status & 1 and done[0].error.startswith("device status"), done[0]
    assert done[1].ok and done[1].status == 0
    alone = Server(cfg)
    r = alone.serve([(0.0, sp[1])])[0]
    alone.close()
    assert np.array_equal(r.delta, done[1].delta)


def test_sort_wait_that_runs_out_reaches_the_caller():
    """The first sort tile of peak 0 never publishes its look-back words, so the next tile's
    bounded wait gives up after a few thousand polls: the step returns, the peak's status has
    bit 1 and pm_get_stats / pm_get_stats_all return 1; peak 1 in the same sort is untouched,
    and with the hook removed the engine sorts correctly again."""
    import ctypes

    from pbh_b200 import _lib
    from pbh_b200.engine import Engine, PeakConfig
    from pbh_b200.ic import recipe_particles
    lib = _lib.load()
    sp = specs(2, sizes=(32,), steps=10)
    ics = [recipe_particles(s) for s in sp]

    def run(stall):
        eng = Engine([PeakConfig(N=32, Np=32, L=1.0), PeakConfig(N=32, Np=32, L=1.0)], graph=False)
        if stall:
            _lib.check(lib.pm_debug_sort_stall(eng._h, 0, 4000), "pm_debug_sort_stall")
        for i, (x, p) in enumerate(ics):
            eng.set_particles(i, x, p, 1.0, mode=_lib.SCHED_RATIO, param=sp[i].ratio(), max_steps=sp[i].steps)
        t0 = time.perf_counter()
        eng.run(3)                                   # the priming sort, then two steps
        eng.sync()
        took = time.perf_counter() - t0
        st = (_lib.StatsInfo * 2)()
        flagged = lib.pm_get_stats_all(eng._h, st)
        one = _lib.StatsInfo()
        rc0 = lib.pm_get_stats(eng._h, 0, ctypes.byref(one))
        out = (flagged, rc0, st[0].status, st[1].status, took, eng.delta(1).cpu().numpy(), eng)
        return out

    flagged, rc0, s0, s1, took, d1, eng = run(stall=True)
    assert flagged == 1 and rc0 == 1 and s0 & 2, (flagged, rc0, s0)
    assert s1 == 0
    assert took < 30.0
    # the context is usable: the hook removed, peak 0 reloaded sorts and steps cleanly
    _lib.check(lib.pm_debug_sort_stall(eng._h, -1, 0), "pm_debug_sort_stall")
    x, p = ics[0]
    eng.set_particles(0, x, p, 1.0, mode=_lib.SCHED_RATIO, param=sp[0].ratio(), max_steps=sp[0].steps)
    eng.run(3)
    assert eng.stats(0).status == 0
    eng.close()
    _, _, c0, c1, _, d1_clean, eng2 = run(stall=False)
    eng2.close()
    assert c0 == 0 and c1 == 0
    assert np.array_equal(d1, d1_clean)              # the stalled peak never touched its neighbour


def test_served_request_fails_on_a_sort_that_gave_up():
    from pbh_b200 import _lib
    from pbh_b200.serve import Server, ServerConfig
    sp = specs(3, sizes=(32,), steps=20)
    srv = Server(ServerConfig(slots={32: 2}, budget_bytes=20e9, delta_collapse=0.0))
    _lib.check(_lib.load().pm_debug_sort_stall(srv._h, 0, 4000), "pm_debug_sort_stall")
    done = {r.rid: r for r in srv.serve([(0.0, sp[0]), (0.0, sp[1])])}
    assert not done[0].ok and done[0].status & 2, done[0]
    assert done[1].ok and done[1].steps == 20
    _lib.check(_lib.load().pm_debug_sort_stall(srv._h, -1, 0), "pm_debug_sort_stall")
    srv.done.clear()
    r = srv.serve([(0.0, sp[2])])[0]                 # slot 0 again, the normal sort
    srv.close()
    assert r.ok and r.slot == 0 and r.status == 0
