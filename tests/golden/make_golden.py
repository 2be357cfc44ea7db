"""Generate the golden fixtures by running the unmodified reference pm3d.

Usage (in a container that has the reference checkout):
    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py <checkout>/pbhgr [pm3d|profiles|collapse ...]

The reference package directory (the one holding pbhgr/ and scripts/ of the reference
checkout) is given on the command line (or through PBH_REFERENCE); the optional names pick
which fixtures to regenerate.  Nothing at test time reads the checkout.  Each case is a small run of
``pbhgr.pm3d`` whose inputs and outputs are saved as float64 ``.npz`` files
(plus ``analyse`` output as JSON), with the numpy version recorded.
"""
from __future__ import annotations

import json
import os
import sys
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _load_reference(path: str):
    sys.path.insert(0, path)
    sys.dont_write_bytecode = True
    warnings.filterwarnings("ignore", category=DeprecationWarning)
    from pbhgr import pm3d, profiles          # noqa: E402
    return pm3d, profiles


def _save(name: str, meta: dict, **arrays):
    meta = dict(meta, numpy=np.__version__)
    np.savez_compressed(HERE / f"{name}.npz", meta=json.dumps(meta), **arrays)


def zeta_case(pm3d, profiles, name, N, L, Np, seed, smooth, mu, e, p, tail, steps):
    """make_ic on the curvature profile, forces at a = 1, a few KDK steps, analyse."""
    spline = profiles.profile_table("yoo")["spline"]
    pm = pm3d.PM3D(N, L, Np, seed=seed, smooth=smooth).make_ic(mu, spline, e, p, tail, (2.0, 10.0))
    ic = dict(x0=pm.x.copy(), p0=pm.p.copy(), delta_lin=pm.delta_lin.copy(), r_ell_q=pm.r_ell_q.copy(),
              A=np.asarray(pm.A),
              # analyse() picks its core sets with a default-kind argsort, whose
              # choice among tied r_ell_q values is numpy's; record it.
              ref_order30=np.argsort(pm.r_ell_q)[:30])
    acc0, delta0 = pm.forces(1.0)
    a = 1.0
    das = []
    for _ in range(steps):
        da = 0.02 * a
        das.append(da)
        a, delta = pm.step(a, da)
    diag = pm3d.analyse(pm, a)
    _save(name, dict(N=N, L=L, Np=Np, seed=seed, smooth=smooth, mu=mu, e=e, p=p, tail=tail, steps=steps,
                     a_end=a, tail_rms_grid=pm.tail_rms_grid, analyse=diag, m_part=pm.m_part),
          acc0=acc0, delta0=delta0, das=np.array(das), x_end=pm.x, p_end=pm.p, delta_end=delta,
          acc_end=pm._acc, **ic)


def mesh_case(pm3d, name, N, L, n, seed):
    """deposit/interp of scattered positions, including cell-face and box-edge points."""
    rng = np.random.default_rng(seed)
    pm = pm3d.PM3D(N, L, 4, seed=0)
    dx = L / N
    X = rng.uniform(0.0, L, size=(n, 3))
    edges = np.array([[0.0, 0.0, 0.0], [L - 1e-12, 0.5 * dx, dx], [0.5 * dx, 1.5 * dx, L - 0.5 * dx],
                      [np.nextafter(L, 0.0), np.nextafter(0.5 * dx, 0.0), np.nextafter(0.5 * dx, 1.0)],
                      [3.25 * dx, 3.75 * dx, 4.5 * dx]])
    X = np.concatenate([X, edges])
    F = rng.standard_normal((N, N, N))
    _save(name, dict(N=N, L=L, seed=seed), X=X, F=F, rho=pm.deposit(X), Fi=pm.interp(F, X))


def recipe_case(pm3d, name, N, Np, seed, steps):
    """The reference step driven from the benchmark-recipe initial condition."""
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle.pm3d_oracle import Mesh
    from oracle.recipe_oracle import recipe_ic
    R = (0.10, 0.09, 0.08)
    delta0 = 0.03
    mesh = Mesh(N, 1.0, Np)
    ic = recipe_ic(mesh, R, delta0, 0.01, seed)
    pm = pm3d.PM3D(N, 1.0, Np, seed=seed)
    pm.x, pm.p = ic["x"].copy(), ic["p"].copy()
    a, fac = 1.0, 100.0 ** (1.0 / 100.0) - 1.0
    snaps = {}
    for s in range(1, steps + 1):
        a, delta = pm.step(a, a * fac)
        if s in (1, steps):
            snaps[f"x_{s}"] = pm.x.copy()
            snaps[f"p_{s}"] = pm.p.copy()
            snaps[f"delta_{s}"] = delta
    _save(name, dict(N=N, Np=Np, seed=seed, R=R, delta0=delta0, noise_frac=0.01, steps=steps, a_end=a),
          x0=ic["x"], p0=ic["p"], **snaps)


def profiles_case(path: str, name="profiles"):
    """Profile tables (pbhgr/pbhgr/profiles.py) and the driver's LTB units (pbhgr/pbhgr/ltb.py)
    used by scripts/pm3d_peak.py: spline values and slopes on a radius grid, r_m, t_H, t_C(0)."""
    sys.path.insert(0, path)
    from pbhgr import ltb, profiles          # noqa: E402
    r = np.linspace(0.0, 20.0, 201)
    out, meta = {}, {}
    for prof in ("yoo", "ln0.5", "ln0.1", "tophat"):
        tab = profiles.profile_table(prof)
        tab["name"] = prof
        key = prof.replace(".", "p")
        out[f"{key}_psi"] = tab["spline"](r)
        out[f"{key}_dpsi"] = tab["spline"].derivative(1)(r)
        for mu in (0.1, 0.5):
            ref = ltb.LTBGaussian(mu) if prof == "yoo" else ltb.LTBProfile(mu, tab)
            tc0 = ref.tC(1e-6)
            if not np.isfinite(tc0):
                tc0 = ref.tC(ref.r_m)
            meta[f"{key}_mu{mu:g}"] = dict(r_m=float(ref.r_m), t_H=float(ref.t_H), tC0=float(tc0))
    _save(name, dict(units=meta), r=r, **out)


COLLAPSE_POINTS = ((0.0, 0.0), (0.05, 0.0), (0.1, -0.05), (0.15, 0.05), (0.2, 0.0), (0.3, 0.1), (0.3, -0.1))


def collapse_case(path: str, name="collapse_times"):
    """Bond-Myers collapse times t1 <= t2 <= t3 of scripts/ellipsoidal_collapse.py (its
    collapse_times, lines 14-54) at a few (e, p) points.  The script runs a scan when it is
    imported, so only its text up to the scan is executed, with the script's default
    arguments (nu = 4, f_freeze = 0.01)."""
    src = Path(path) / "scripts" / "ellipsoidal_collapse.py"
    text = src.read_text()
    head = text[:text.index("\nt_sph = collapse_times")]
    ns = {"__name__": "ellipsoidal_collapse_defs"}
    argv = sys.argv
    sys.argv = [str(src)]
    try:
        exec(compile(head, str(src), "exec"), ns)
    finally:
        sys.argv = argv
    times = np.array([ns["collapse_times"](e, p) for e, p in COLLAPSE_POINTS])
    _save(name, dict(f_freeze=ns["f_freeze"], delta_i=1e-2, points=[list(q) for q in COLLAPSE_POINTS]),
          ep=np.array(COLLAPSE_POINTS), times=times)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PBH_REFERENCE", "")
    if not ref:
        raise SystemExit("give the reference package directory (the one holding pbhgr/)")
    only = sys.argv[2:]
    if not only or "pm3d" in only:
        pm3d, profiles = _load_reference(ref)
        zeta_case(pm3d, profiles, "zeta_16", 16, 8.0, 16, 7, 0.0, 0.1, 0.15, 0.05, 0.05, 3)
        zeta_case(pm3d, profiles, "zeta_16_np8_smooth", 16, 8.0, 8, 1, 2.0, 0.3, 0.0, 0.0, 0.0, 4)
        mesh_case(pm3d, "mesh_8", 8, 1.0, 600, 11)
        recipe_case(pm3d, "recipe_16", 16, 16, 5, 10)
    if not only or "profiles" in only:
        profiles_case(ref)
    if not only or "collapse" in only:
        collapse_case(ref)


if __name__ == "__main__":
    main()
