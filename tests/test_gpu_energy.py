"""Energy and momentum sums of the engine (compensated FP64, sampled every step) against the
float64 oracle: the same quantities on the oracle's own trajectory from the same particles,
and the Layzer-Irvine residual a (K + W) + int K da - a0 (K0 + W0) accumulated the same way."""
import numpy as np
import pytest

from oracle import pm3d_oracle as O
from oracle.recipe_oracle import recipe_ic

pytestmark = pytest.mark.gpu

RATIO = (100.0 ** (1.0 / 100.0)) - 1.0     # 100 steps uniform in ln a over a factor 100


def test_energy_and_layzer_irvine_match_oracle():
    from pbh_b200._lib import SCHED_RATIO, STATE_IDLE
    from pbh_b200.engine import Engine, PeakConfig
    N, nsteps = 32, 20
    mesh = O.Mesh(N, 1.0, N)
    ic = recipe_ic(mesh, R=(0.10, 0.09, 0.08), delta0=0.5, noise_frac=0.01, seed=5)
    eng = Engine([PeakConfig(N=N, Np=N, L=1.0)])
    eng.set_particles(0, ic["x"], ic["p"], 1.0, mode=SCHED_RATIO, param=RATIO, max_steps=nsteps)
    x0, p0 = [t.cpu().numpy() for t in eng.particles(0)]
    eng.run(nsteps + 2)                                  # prime + steps + closing kick
    assert eng.clock(0).state == STATE_IDLE
    s = eng.stats(0)
    assert s.energy_samples == nsteps + 1
    tr = O.Trajectory(mesh, x0, p0)
    a = 1.0
    samples = []
    mom, kin, pot = O.energies(mesh, tr.x, tr.p, a)
    samples.append((a, kin, pot))
    for _ in range(nsteps):
        a, _ = tr.step(a, a * RATIO)
        mom, kin, pot = O.energies(mesh, tr.x, tr.p, a)
        samples.append((a, kin, pot))
    assert abs(s.a_energy - a) < 1e-12
    assert abs(s.kinetic - kin) <= 1e-4 * abs(kin)
    assert abs(s.potential - pot) <= 1e-4 * abs(pot)
    scale = a * (kin + abs(pot))
    assert abs(s.li_scale - scale) <= 1e-4 * scale
    li = O.layzer_irvine(samples)
    # the engine's residual is the oracle's, up to the FP32 trajectory gap
    assert abs(s.li_residual - li) <= 1e-4 * scale
    # total momentum stays at its (near-zero) start: compare with the momentum scale m_p n |p|_rms
    pscale = np.sqrt(2.0 * kin * a * a * mesh.m_part * mesh.Np ** 3)
    assert np.max(np.abs(np.array(list(s.momentum)) - mom)) <= 1e-5 * pscale


def test_energy_at_loaded_positions():
    """First sample: K, W and the momentum of the loaded particles at a0."""
    from pbh_b200._lib import SCHED_RATIO
    from pbh_b200.engine import Engine, PeakConfig
    N = 16
    mesh = O.Mesh(N, 1.0, N)
    ic = recipe_ic(mesh, R=(0.12, 0.1, 0.09), delta0=0.3, noise_frac=0.02, seed=2)
    eng = Engine([PeakConfig(N=N, Np=N, L=1.0, tile=8)], graph=False)
    eng.set_particles(0, ic["x"], ic["p"], 1.0, mode=SCHED_RATIO, param=0.01, max_steps=5)
    x0, p0 = [t.cpu().numpy() for t in eng.particles(0)]
    eng.run(2)                                           # prime, then the first push samples a0
    s = eng.stats(0)
    assert s.energy_samples == 1 and s.a_energy == 1.0
    mom, kin, pot = O.energies(mesh, x0, p0, 1.0)
    assert abs(s.kinetic - kin) <= 1e-6 * abs(kin)
    assert abs(s.potential - pot) <= 1e-5 * abs(pot)
    assert abs(s.li_residual) <= 1e-12 * s.li_scale
