"""The drop-in PM3D (pbh_b200.pm3d) against the reference's own golden runs and the oracle."""
import numpy as np
import pytest
from scipy.interpolate import CubicSpline

from oracle import pm3d_oracle as O
from oracle.recipe_oracle import recipe_ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def wrap(d, L):
    return (d + L / 2) % L - L / 2


def yoo_spline():
    # profile 'yoo' of pbhgr/pbhgr/profiles.py:52-53,60
    r = np.linspace(0.0, 40.0, 4001)
    return CubicSpline(r, np.exp(-r ** 2 / 6), bc_type=((1, 0.0), (1, 0.0)))


@pytest.mark.parametrize("case", ["zeta_16", "zeta_16_np8_smooth"])
def test_make_ic_forces_steps_vs_reference(golden, case):
    from pbh_b200.pm3d import PM3D
    g = golden(case)
    m = g["meta"]
    pm = PM3D(m["N"], m["L"], m["Np"], seed=m["seed"], smooth=m["smooth"])
    pm.keep_ic = True
    pm.make_ic(m["mu"], yoo_spline(), m["e"], m["p"], m["tail"], (2.0, 10.0))
    # the float64 device IC itself
    x_ic, p_ic = [t.cpu().numpy() for t in pm._ic_xp]
    assert rel(x_ic, g["x0"]) < 1e-12
    assert rel(p_ic, g["p0"]) < 1e-12
    assert rel(pm.delta_lin, g["delta_lin"]) < 1e-12
    assert abs(pm.tail_rms_grid - m["tail_rms_grid"]) <= 1e-12 * max(1.0, m["tail_rms_grid"])
    assert rel(pm.r_ell_q, g["r_ell_q"]) < 1e-14
    # stored as int32 cell + FP32 offset / FP32 momentum
    dx = m["L"] / m["N"]
    assert np.max(np.abs(wrap(pm.x - g["x0"], m["L"]))) / dx < 1e-6
    assert rel(pm.p, g["p0"]) < 1e-6
    acc, delta = pm.forces(1.0)
    # against the reference's own float64 positions: FP32 offsets move particles by ~1e-8 cells,
    # which shifts a delta of rms ~1e-4 by ~1e-5 relative; the same-position checks below gate.
    assert rel(acc, g["acc0"]) < 1e-4
    assert rel(delta, g["delta0"]) < 1e-4
    mesh = O.Mesh(m["N"], m["L"], m["Np"], m["smooth"])
    xg = pm.x
    acc_o, delta_o = O.accelerations(mesh, xg, 1.0)        # same positions: kernel tolerances
    assert rel(acc, acc_o) < 1e-5
    assert rel(delta, delta_o) < 1e-6
    a = 1.0
    for da in g["das"]:
        a, delta = pm.step(a, da)
    assert abs(a - m["a_end"]) < 1e-14
    assert np.max(np.abs(wrap(pm.x - g["x_end"], m["L"]))) / dx < 1e-5
    assert rel(pm.p, g["p_end"]) < 1e-5
    assert rel(pm._acc, g["acc_end"]) < 1e-4
    assert pm._acc_a == a
    assert rel(delta, O.density_contrast(mesh, pm.x)) < 1e-6


def test_analyse_matches_oracle_on_same_positions(golden):
    from pbh_b200.pm3d import PM3D, analyse
    g = golden("zeta_16")
    m = g["meta"]
    pm = PM3D(m["N"], m["L"], m["Np"], seed=m["seed"])
    pm.make_ic(m["mu"], yoo_spline(), m["e"], m["p"], m["tail"], (2.0, 10.0))
    a = 1.0
    for da in g["das"]:
        a, _ = pm.step(a, da)
    d = analyse(pm, a)
    mesh = O.Mesh(m["N"], m["L"], m["Np"])
    ref = O.analyse(mesh, pm.x, pm.r_ell_q, a)             # stable tie order, like the product
    for k, v in ref.items():
        assert np.allclose(d[k], v, rtol=1e-9, atol=1e-12), (k, d[k], v)
    # keys that do not depend on the tie order agree with the reference run itself
    for k in ("M_0.1", "M_0.2", "M_0.3", "rho_max_over_mean"):
        assert np.allclose(d[k], m["analyse"][k], rtol=1e-5), k


def test_recipe_peak_and_deposit_interp(golden):
    from pbh_b200.pm3d import PM3D
    N = 32
    pm = PM3D(N, 1.0, N, seed=4)
    pm.keep_ic = True
    pm.make_peak((0.10, 0.09, 0.08), 0.02, 0.01)
    mesh = O.Mesh(N, 1.0, N)
    ic = recipe_ic(mesh, (0.10, 0.09, 0.08), 0.02, 0.01, 4)
    x_ic, p_ic = [t.cpu().numpy() for t in pm._ic_xp]
    assert rel(x_ic, ic["x"]) < 1e-12
    assert rel(p_ic, ic["p"]) < 1e-12
    gm = golden("mesh_8")
    pm8 = PM3D(8, 1.0, 4)
    rho = pm8.deposit(gm["X"])
    # float64 offsets, each corner weight rounded to 2^-39 of a particle: the reference's counts
    # to ~1e-12, mass exact, and the same bits for the positions in any order
    assert rel(rho, gm["rho"]) < 1e-11
    assert rho.sum() == len(gm["X"])
    perm = np.random.default_rng(1).permutation(len(gm["X"]))
    assert np.array_equal(pm8.deposit(gm["X"][perm]), rho)
    assert rel(pm8.interp(gm["F"], gm["X"]), gm["Fi"]) < 1e-14
    # no particles: zero counts and an empty gather, as the reference's bincount and indexing give
    empty = np.empty((0, 3))
    rho0 = pm8.deposit(empty)
    assert rho0.shape == (8, 8, 8) and not rho0.any()
    assert pm8.interp(gm["F"], empty).shape == (0,)


def test_run_loop_matches_explicit_steps():
    from pbh_b200.pm3d import PM3D
    N = 16
    a_end, frac = 1.6, 0.05
    pa = PM3D(N, 1.0, N, seed=2).make_peak((0.1, 0.09, 0.08), 0.05)
    pb = PM3D(N, 1.0, N, seed=2).make_peak((0.1, 0.09, 0.08), 0.05)
    a = 1.0
    while a < a_end:                                      # pbhgr/scripts/pm3d_peak.py:26-28
        a, _ = pa.step(a, min(frac * a, a_end - a))
    ab = pb.run(a_end, frac)
    assert abs(ab - a) < 1e-12
    assert np.max(np.abs(wrap(pa.x - pb.x, 1.0))) < 1e-12
    assert rel(pa.p, pb.p) < 1e-6


def test_writing_into_x_and_p_changes_the_run():
    """pm.x / pm.p are plain arrays in the reference (pm3d.py:67-68); writing into them must
    change the next step here too, exactly as assigning the modified arrays does."""
    from pbh_b200.pm3d import PM3D
    N = 16
    pa = PM3D(N, 1.0, N, seed=5).make_peak((0.1, 0.09, 0.08), 0.05)
    pb = PM3D(N, 1.0, N, seed=5).make_peak((0.1, 0.09, 0.08), 0.05)
    a, _ = pa.step(1.0, 0.05)
    pb.step(1.0, 0.05)
    pa.p[:, 0] *= 2.0                                    # in place, through the property
    pa.x[7] = (0.5, 0.25, 0.125)
    p_new, x_new = pb.p.copy(), pb.x.copy()
    p_new[:, 0] *= 2.0
    x_new[7] = (0.5, 0.25, 0.125)
    pb.p = p_new                                         # assignment
    pb.x = x_new
    # pa holds its written float64 copies until its next device operation, pb's were loaded
    # (momenta in FP32): equal to FP32 rounding here, bit for bit once both are on the device
    assert np.array_equal(pa.x, pb.x)
    assert np.allclose(pa.p, pb.p, rtol=1e-6, atol=0.0)
    ra = pa.step(a, 0.05)[1]
    rb = pb.step(a, 0.05)[1]
    assert np.array_equal(ra, rb)
    assert np.array_equal(pa.x, pb.x) and np.array_equal(pa.p, pb.p)
    assert abs(pa.x[7, 0] - 0.5) > 0.0                   # it moved from the written position
    stale = pa.x
    pa.step(a + 0.05, 0.05)
    stale[0] = 0.0                                       # a copy from before the step: no effect
    assert not np.array_equal(pa.x[0], np.zeros(3))
