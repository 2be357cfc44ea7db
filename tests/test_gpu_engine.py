"""GPU parity of the native engine against the CPU oracle (same inputs, seeded)."""
import numpy as np
import pytest

from oracle import pm3d_oracle as O
from oracle.recipe_oracle import recipe_ic

pytestmark = pytest.mark.gpu

# Tolerances of the path: relative L2 for density and forces, cells for positions.
TOL_DENSITY = 1e-6
TOL_FORCE = 1e-5
TOL_POS_CELLS = 1e-5
RATIO_100 = 100.0 ** (1.0 / 100.0) - 1.0   # 100 steps uniform in ln a over a factor 100


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def wrap(d, L):
    return (d + L / 2) % L - L / 2


def recipe(N, Np=None, seed=1, delta0=0.02):
    mesh = O.Mesh(N, 1.0, Np or N)
    return mesh, recipe_ic(mesh, (0.10, 0.09, 0.08), delta0, 0.01, seed)


def engine(cfgs, **kw):
    from pbh_b200.engine import Engine, PeakConfig
    return Engine([PeakConfig(**c) for c in cfgs], **kw)



def test_sort_matches_numpy_stable():
    from pbh_b200.engine import sort_u64
    rng = np.random.default_rng(0)
    cases = [(1, 0, 64), (4097, 0, 64), (100003, 0, 64), (300000, 3, 27), (70000, 0, 12), (8192, 40, 64)]
    for n, lo, hi in cases:
        keys = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64)
        keys[::3] = keys[0]                                # many exact ties
        keys[1::7] &= np.uint64(0xFFFF)                    # clustered small keys
        ks, perm = sort_u64(keys, lo, hi)
        span = hi - lo
        masked = keys >> np.uint64(lo)
        if span < 64:
            masked &= np.uint64((1 << span) - 1)
        ref = np.argsort(masked, kind="stable")
        assert np.array_equal(perm.astype(np.int64), ref), (n, lo, hi)
        assert np.array_equal(ks, keys[ref]), (n, lo, hi)


def test_interp64_matches_oracle(golden):
    from pbh_b200.engine import interp64
    g = golden("mesh_8")
    m = g["meta"]
    out = interp64(g["F"], g["X"], m["L"]).cpu().numpy()
    assert rel(out, g["Fi"]) < 1e-14


# (32, 64, 16): 32.8k particles per super-tile, so the deposit folds several chunks.
@pytest.mark.parametrize("N,Np,tile", [(32, 32, 16), (32, 32, 8), (16, 8, 4), (64, 64, 16), (64, 48, 0), (64, 64, 4),
                                       (32, 64, 16)])
def test_deposit_forces_same_positions(N, Np, tile):
    mesh, ic = recipe(N, Np)
    eng = engine([dict(N=N, Np=Np, L=1.0, tile=tile)])
    eng.set_particles(0, ic["x"], ic["p"], 1.0)
    eng.run(1)                                           # prime: sort, deposit, forces at a = 1
    x, _ = eng.particles(0)
    x = x.cpu().numpy()
    assert np.max(np.abs(wrap(x - ic["x"], 1.0))) / mesh.dx < 1e-6
    counts = eng.counts(0).cpu().numpy()
    ref = O.deposit(x, N, mesh.dx)
    # fixed point with 38 fractional bits: each corner weight is rounded to 2^-39 of a particle
    assert rel(counts, ref) < 5e-11
    delta = eng.delta(0).cpu().numpy()
    ref_delta = ref / mesh.n_mean - 1.0
    assert rel(delta, ref_delta) < TOL_DENSITY
    acc = eng.acc(0, 1.0).cpu().numpy()
    ref_acc, _ = O.accelerations(mesh, x, 1.0)
    assert rel(acc, ref_acc) < TOL_FORCE
    acc3 = eng.acc(0, 3.0).cpu().numpy()                 # forces(a) at another a rescales 1/a
    ref_acc3, _ = O.accelerations(mesh, x, 3.0)
    assert rel(acc3, ref_acc3) < TOL_FORCE
    s = eng.stats(0)
    assert s.mass_defect == 0.0 and s.status == 0
    assert abs(s.rho_max_over_mean - ref.max() / mesh.n_mean) < 1e-9


@pytest.mark.parametrize("graph", [True, False])
def test_trajectory_50_steps(graph):
    from pbh_b200._lib import SCHED_RATIO, STATE_IDLE
    N = 32
    mesh, ic = recipe(N, delta0=0.03)
    eng = engine([dict(N=N, Np=N, L=1.0)], graph=graph)
    eng.set_particles(0, ic["x"], ic["p"], 1.0, mode=SCHED_RATIO, param=RATIO_100, max_steps=50)
    x0, p0 = [t.cpu().numpy() for t in eng.particles(0)]
    eng.run(52)                                          # prime + 50 steps + closing kick
    c = eng.clock(0)
    assert c.state == STATE_IDLE and c.nsteps == 50
    x, p = [t.cpu().numpy() for t in eng.particles(0)]
    tr = O.Trajectory(mesh, x0, p0)
    a = 1.0
    for _ in range(50):
        a, delta = tr.step(a, a * RATIO_100)
    assert abs(c.a - a) < 1e-12
    assert np.max(np.abs(wrap(x - tr.x, 1.0))) / mesh.dx < TOL_POS_CELLS
    assert rel(p, tr.p) < 1e-4
    d = eng.delta(0).cpu().numpy()
    assert rel(d, delta) < 1e-4                          # trajectory gap, reported not gated tightly
    # the GPU's own final positions give the oracle's density within the kernel tolerance
    assert rel(d, O.density_contrast(mesh, x)) < TOL_DENSITY
    s = eng.stats(0)
    assert s.mass_defect == 0.0 and s.status == 0


def test_explicit_steps_match_oracle():
    N = 16
    mesh, ic = recipe(N, delta0=0.05, seed=3)
    eng = engine([dict(N=N, Np=N, L=1.0, tile=4)])
    eng.set_particles(0, ic["x"], ic["p"], 1.0)
    x0, p0 = [t.cpu().numpy() for t in eng.particles(0)]
    tr = O.Trajectory(mesh, x0, p0)
    a = 1.0
    for _ in range(4):
        da = 0.05 * a
        eng.step_explicit(0, a, da)
        a, delta = tr.step(a, da)
    x, p = [t.cpu().numpy() for t in eng.particles(0)]
    assert np.max(np.abs(wrap(x - tr.x, 1.0))) / mesh.dx < TOL_POS_CELLS
    assert rel(p, tr.p) < 1e-5
    d = eng.delta(0).cpu().numpy()
    assert rel(d, delta) < 1e-4                          # trajectory gap (FP32 positions)
    assert rel(d, O.density_contrast(mesh, x)) < TOL_DENSITY
    # a step that does not continue from the current a recomputes the forces (pm3d.py:119)
    eng.step_explicit(0, 2.0 * a, 0.01)
    a2, d2 = tr.step(2.0 * a, 0.01)
    x, p = [t.cpu().numpy() for t in eng.particles(0)]
    assert np.max(np.abs(wrap(x - tr.x, 1.0))) / mesh.dx < TOL_POS_CELLS
    assert rel(p, tr.p) < 1e-5


def test_deposit_is_order_independent_bitwise():
    N = 32
    mesh, ic = recipe(N)
    perm = np.random.default_rng(9).permutation(N ** 3)
    outs = []
    for order in (np.arange(N ** 3), perm):
        eng = engine([dict(N=N, Np=N, L=1.0)])
        eng.set_particles(0, ic["x"][order], ic["p"][order], 1.0)
        eng.run(1)
        outs.append(eng.delta(0).cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_batched_peaks_equal_alone():
    from pbh_b200._lib import SCHED_RATIO
    specs = [(16, 2), (32, 5), (16, 7)]
    ics = [recipe(N, seed=s, delta0=0.04)[1] for N, s in specs]
    mix = engine([dict(N=N, Np=N, L=1.0) for N, _ in specs])
    for i, ic in enumerate(ics):
        mix.set_particles(i, ic["x"], ic["p"], 1.0, mode=SCHED_RATIO, param=RATIO_100, max_steps=5 + 3 * i)
    mix.run(20)
    for i, ((N, _), ic) in enumerate(zip(specs, ics)):
        alone = engine([dict(N=N, Np=N, L=1.0)])
        alone.set_particles(0, ic["x"], ic["p"], 1.0, mode=SCHED_RATIO, param=RATIO_100, max_steps=5 + 3 * i)
        alone.run(20)
        xa, pa = [t.cpu().numpy() for t in alone.particles(0)]
        xm, pm = [t.cpu().numpy() for t in mix.particles(i)]
        assert np.array_equal(xa, xm) and np.array_equal(pa, pm), i
        assert np.array_equal(alone.delta(0).cpu().numpy(), mix.delta(i).cpu().numpy()), i


@pytest.mark.parametrize("Np,tile", [(32, 8), (48, 16)])
def test_refresh_every_step_equals_every_16th(Np, tile):
    """Bins kept by the push with the per-super-tile re-sort every step or every 16th step give
    the same run, bit for bit (the order inside a super-tile never changes a result).  Np = 48 on
    a 32^3 mesh with 16^3 super-tiles puts ~13.8k particles in each super-tile, beyond the
    shared-memory capacity of the re-sort (5120), so its global-memory path runs too."""
    from pbh_b200._lib import SCHED_RATIO
    N = 32
    mesh, ic = recipe(N, Np, delta0=0.05, seed=8)
    runs = []
    for every in (1, 16):
        eng = engine([dict(N=N, Np=Np, L=1.0, tile=tile)], full_every=every)
        eng.set_particles(0, ic["x"], ic["p"], 1.0, mode=SCHED_RATIO, param=RATIO_100, max_steps=20)
        eng.run(22)
        x, p = [t.cpu().numpy() for t in eng.particles(0)]
        runs.append((x, p, eng.delta(0).cpu().numpy()))
        s = eng.stats(0)
        assert s.mass_defect == 0.0 and s.status == 0
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("N,Np,tile,pscale,fast", [(32, 32, 8, 3.0, 1.0), (32, 48, 16, 3.0, 1.0), (64, 32, 4, 6.0, 1.0),
                                                    (32, 32, 8, 3.0, 0.002), (64, 64, 16, 3.0, 0.0005)])
def test_overflowing_bins_relayout_without_changing_results(N, Np, tile, pscale, fast):
    """Bins without spare capacity overflow on almost every step once particles cross super-tile
    faces (random positions; a fraction `fast` of them with momenta drifting about a cell per
    step, the rest at rest).  Each overflow sends the peak through a relayout: the overflowed
    bins move to free space after the last bin when it holds them (partial), else every bin is
    laid out again and copied to the other buffer (full).  With every particle fast the bins all
    overflow and the relayouts are full; with a few fast ones most are partial.  Positions,
    momenta and delta stay the same bit for bit as with the normal spare capacity, and the mass
    stays exact.  Np = 48 with 16^3 super-tiles also takes the global-memory paths of the
    super-tile re-sort and of the deposit (more than one chunk)."""
    from pbh_b200._lib import SCHED_RATIO
    rng = np.random.default_rng(31)
    x = rng.uniform(0.0, 1.0, size=(Np ** 3, 3))
    p = rng.normal(0.0, pscale, size=(Np ** 3, 3))
    p[rng.uniform(size=Np ** 3) >= fast] = 0.0
    runs, counts = [], []
    for tight in (False, True):
        eng = engine([dict(N=N, Np=Np, L=1.0, tile=tile)], tight_bins=tight, full_every=16)
        eng.set_particles(0, x, p, 1.0, mode=SCHED_RATIO, param=RATIO_100, max_steps=20)
        eng.run(22)
        xg, pg = [t.cpu().numpy() for t in eng.particles(0)]
        runs.append((xg, pg, eng.delta(0).cpu().numpy()))
        s = eng.stats(0)
        assert s.mass_defect == 0.0 and s.status == 0, (tight, s.status)
        counts.append((s.relayouts, s.relayouts_full))
        eng.close()
    relayouts, full = counts[1]
    assert relayouts >= 10, counts                # tight bins: most steps relayout
    if fast == 1.0:
        assert full >= 1, counts                  # every bin overflows: no room for a partial move
    else:
        assert relayouts - full >= 1, counts      # a few bins overflow: moved after the last bin
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)


def test_converging_flow_piles_particles_into_few_super_tiles():
    """Momenta pointing at the box centre move most particles into the few central super-tiles
    within five steps: their bins grow ten times over and more (relayouts with large
    capacities).  Positions after each step against the float64 oracle, exact mass,
    and the pile-up itself."""
    N, Np = 32, 32
    mesh = O.Mesh(N, 1.0, Np)
    rng = np.random.default_rng(41)
    x = rng.uniform(0.0, 1.0, size=(Np ** 3, 3))
    p = -(x - 0.5) * 26.0                                 # about a fifth of the way in per step
    eng = engine([dict(N=N, Np=Np, L=1.0, tile=8)])        # 4 super-tiles per axis, 512 particles each
    eng.set_particles(0, x, p, 1.0)
    x0, p0 = [t.cpu().numpy() for t in eng.particles(0)]
    tr = O.Trajectory(mesh, x0, p0)
    a = 1.0
    for _ in range(5):
        eng.step_explicit(0, a, 0.05)
        a, delta = tr.step(a, 0.05)
        xg = eng.particles(0)[0].cpu().numpy()
        assert np.max(np.abs(wrap(xg - tr.x, 1.0))) / mesh.dx < TOL_POS_CELLS
    s = eng.stats(0)
    assert s.mass_defect == 0.0 and s.status == 0
    assert s.relayouts >= 1
    tiles = np.floor(((xg / mesh.dx - 0.5) % N) / 8).astype(int)
    counts = np.bincount((tiles[:, 0] * 4 + tiles[:, 1]) * 4 + tiles[:, 2], minlength=64)
    assert counts.max() >= 8 * Np ** 3 // 64               # the central bins hold many times their share
    assert rel(eng.delta(0).cpu().numpy(), O.density_contrast(mesh, xg)) < TOL_DENSITY


def test_fast_particles_cross_several_super_tiles():
    """Particles that move more than two super-tiles in one step land in their new bins."""
    N, Np = 64, 16
    mesh = O.Mesh(N, 1.0, Np)
    rng = np.random.default_rng(21)
    x = rng.uniform(0.0, 1.0, size=(Np ** 3, 3))
    p = rng.normal(0.0, 1.0, size=(Np ** 3, 3)) * 8.0      # drifts of up to ~25 cells in one step
    eng = engine([dict(N=N, Np=Np, L=1.0, tile=4)])       # 16 super-tiles per axis
    eng.set_particles(0, x, p, 1.0)
    x0, p0 = [t.cpu().numpy() for t in eng.particles(0)]
    tr = O.Trajectory(mesh, x0, p0)
    a = 1.0
    for _ in range(2):
        eng.step_explicit(0, a, 0.05)
        a, delta = tr.step(a, 0.05)
    xg, pg = [t.cpu().numpy() for t in eng.particles(0)]
    moved = np.max(np.abs(wrap(xg - x0, 1.0))) / mesh.dx
    assert moved > 12.0                                   # some particle crossed > 2 super-tiles
    assert np.max(np.abs(wrap(xg - tr.x, 1.0))) / mesh.dx < TOL_POS_CELLS
    assert rel(eng.delta(0).cpu().numpy(), O.density_contrast(mesh, xg)) < TOL_DENSITY
    s = eng.stats(0)
    assert s.mass_defect == 0.0 and s.status == 0


@pytest.mark.parametrize("gradient,order", [("fd2", 2), ("fd4", 4)])
def test_finite_difference_gradients(gradient, order):
    """The engine's finite-difference gradients (transfer functions sin(k dx)/dx and
    (8 sin(k dx) - sin(2 k dx))/(6 dx) applied in k-space) against central differences of the
    oracle's potential taken in real space, at the same positions."""
    N = 32
    mesh, ic = recipe(N, delta0=0.1, seed=4)
    eng = engine([dict(N=N, Np=N, L=1.0, gradient=gradient)])
    eng.set_particles(0, ic["x"], ic["p"], 1.0)
    eng.run(1)
    x = eng.particles(0)[0].cpu().numpy()
    delta = O.density_contrast(mesh, x)
    grids = O.force_grids_fd(mesh, delta, 1.0, order)
    ref = np.stack([O.interp(g, x, N, mesh.dx) for g in grids], axis=-1)
    acc = eng.acc(0, 1.0).cpu().numpy()
    assert rel(acc, ref) < TOL_FORCE
    spectral, _ = O.accelerations(mesh, x, 1.0)
    assert rel(ref, spectral) > 1e-3                      # the stencils differ from the spectral gradient


def test_batched_mix_of_benchmark_sizes_equals_alone():
    """The batched ensemble's own mesh sizes (32^3-256^3, two peaks of the smallest sizes so
    their classes are batched transforms, super-tiles as the bench picks them) against every
    peak alone: positions, momenta and density identical, bit for bit, over 20 steps (one
    refresh of the super-tile order included)."""
    from pbh_b200 import recipe
    from pbh_b200.batch import Ensemble
    tiles = {32: 8, 64: 8, 128: 16, 256: 16}
    pool = recipe.ensemble(npeaks=24, sizes=(32, 64, 128, 256), steps=150, seed=77)
    want = {32: 2, 64: 2, 128: 1, 256: 1}
    specs = []
    for s in pool:
        if want.get(s.N, 0):
            specs.append(s)
            want[s.N] -= 1
    assert not any(want.values())
    mix = Ensemble(specs, tiles=tiles)
    mix.load()
    mix.step(21)
    got = [(*[t.cpu().numpy() for t in mix.engine.particles(i)], mix.engine.delta(i).cpu().numpy())
           for i in range(len(specs))]
    assert all(s.status == 0 and s.mass_defect == 0.0 for s in mix.stats())
    mix.close()
    for i, s in enumerate(specs):
        alone = Ensemble([s], tiles=tiles)
        alone.load()
        alone.step(21)
        xa, pa = [t.cpu().numpy() for t in alone.engine.particles(0)]
        da = alone.engine.delta(0).cpu().numpy()
        alone.close()
        assert np.array_equal(xa, got[i][0]) and np.array_equal(pa, got[i][1]), (i, s.N)
        assert np.array_equal(da, got[i][2]), (i, s.N)
