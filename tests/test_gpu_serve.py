"""Served runs: continuous batching, admission by budget, and results independent of the mix."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_DENSITY = 1e-6


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, float) - np.asarray(b, float)) / max(np.linalg.norm(b), 1e-300))


def specs(n, steps=40, seed=11):
    from pbh_b200 import recipe
    # early collapse times so the short runs cross the threshold
    return recipe.ensemble(npeaks=n, sizes=(16, 32), steps=steps, seed=seed, a_range=(0.02, 0.05))


def test_device_noise_is_seeded_standard_normal():
    import torch

    from pbh_b200.ic import KIND_GAUSS, make_particles
    a = make_particles(32, 32, 1.0, KIND_GAUSS, 0.02, (0.1, 0.09, 0.08), noise_frac=0.01, noise_seed=5)
    b = make_particles(32, 32, 1.0, KIND_GAUSS, 0.02, (0.1, 0.09, 0.08), noise_frac=0.01, noise_seed=5)
    c = make_particles(32, 32, 1.0, KIND_GAUSS, 0.02, (0.1, 0.09, 0.08), noise_frac=0.01, noise_seed=6)
    assert torch.equal(a[0], b[0]) and not torch.equal(a[0], c[0])


def test_served_results_equal_alone():
    from pbh_b200.serve import Server, ServerConfig
    sp = specs(6)
    cfg = ServerConfig(slots={16: 3, 32: 3}, budget_bytes=50e9, delta_collapse=2.0)
    srv = Server(cfg)
    arrivals = [(0.0, sp[0]), (0.0, sp[1]), (0.05, sp[2]), (0.1, sp[3]), (0.1, sp[4]), (0.2, sp[5])]
    done = {r.rid: r for r in srv.serve(arrivals)}
    srv.close()
    assert len(done) == len(sp)
    for i, s in enumerate(sp):
        alone = Server(ServerConfig(slots={s.N: 1}, budget_bytes=50e9, delta_collapse=2.0))
        r = alone.serve([(0.0, s)])[0]
        alone.close()
        m = done[i]
        assert m.steps == r.steps, i
        assert m.a_collapse_cfg == r.a_collapse_cfg, i
        assert np.array_equal(m.delta, r.delta), i      # the deposit sums integers: same bits


def test_served_benchmark_sizes_equal_alone():
    """The served stream's own mesh sizes (64^3-256^3): six requests arriving while others run,
    each result (steps, collapse a, final density) identical to the same request served alone."""
    from pbh_b200 import recipe
    from pbh_b200.serve import Server, ServerConfig
    sp = recipe.ensemble(npeaks=6, sizes=(64, 128, 256), steps=40, seed=29, a_range=(0.03, 0.06))
    cfg = ServerConfig(slots={64: 2, 128: 2, 256: 1}, budget_bytes=60e9, delta_collapse=2.0)
    srv = Server(cfg)
    arrivals = [(0.02 * i, s) for i, s in enumerate(sp)]
    done = {r.rid: r for r in srv.serve(arrivals)}
    srv.close()
    assert len(done) == len(sp) and all(r.ok for r in done.values())
    for i, s in enumerate(sp):
        alone = Server(ServerConfig(slots={s.N: 1}, budget_bytes=60e9, delta_collapse=2.0))
        r = alone.serve([(0.0, s)])[0]
        alone.close()
        m = done[i]
        assert m.steps == r.steps and m.a_collapse_cfg == r.a_collapse_cfg, (i, s.N)
        assert np.array_equal(m.delta, r.delta), (i, s.N)


def test_admission_waits_for_free_slots():
    from pbh_b200.serve import Server, ServerConfig, latency_summary
    sp = specs(5, steps=12)
    srv = Server(ServerConfig(slots={16: 1, 32: 1}, budget_bytes=50e9, delta_collapse=0.0))
    done = srv.serve([(0.0, s) for s in sp])
    srv.close()
    assert len(done) == 5
    assert all(r.steps == 12 for r in done)
    # one slot per size: at most one run of each size at a time -- the next run of a size is
    # primed by a step after the one its predecessor ended on (its result may still be on its
    # way to the host then: the slot is reused as soon as the device is done with it)
    for N in (16, 32):
        rs = sorted((r for r in done if r.spec.N == N), key=lambda r: r.admit_step)
        for a, b in zip(rs, rs[1:]):
            assert b.admit_step > a.end_step >= a.admit_step, (a.admit_step, a.end_step, b.admit_step)
            assert b.t_admit >= a.t_admit
    s = latency_summary(done)
    assert s["completed"] == 5 and s["p99_s"] >= s["p50_s"] > 0


@pytest.mark.parametrize("sizes", [[64, 64, 64], [128, 128], [256]])
def test_slot_footprint_matches_the_engine_allocation(sizes):
    """The admission budget counts serve.slot_bytes per slot; the served engine's own device
    allocation (dynamic mode, native transform where it applies) stays within 5 % of it."""
    from pbh_b200.engine import Engine, PeakConfig
    from pbh_b200.serve import slot_bytes
    eng = Engine([PeakConfig(N=n, Np=n, L=1.0) for n in sizes], graph=False, dynamic=True)
    try:
        got = eng.device_bytes
    finally:
        eng.close()
    est = sum(slot_bytes(n) for n in sizes)
    assert 0.95 * est <= got <= 1.05 * est, (got, est)
