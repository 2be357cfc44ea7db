"""Benchmark peak recipes (host-side set-up of initial-condition parameters).

A recipe peak is a Gaussian linear density field delta0 exp(-sum x_i^2/2R_i^2) in a periodic
box of side L, at the start a_cfg = 0.01 of a run to a_cfg = 1 (pm3d units a = 100 a_cfg, so
a in [1, 100]), plus seeded k^-2 noise at 1% of delta0.  delta0 is fixed by linear theory so
that the peak's first (shortest) axis collapses at a chosen a_cfg:

    delta0 = 1.686 * (t1/t_sph)^(2/3) / a_c,pm

where t1/t_sph is the Bond & Myers (1996) homogeneous-ellipsoid first-axis collapse time in
units of the spherical one for the peak's Zel'dovich (e, p) -- the model of
pbhgr/scripts/ellipsoidal_collapse.py:14-54, restated below -- and 1.686 is the linear
spherical-collapse threshold.  The triaxial shape is either given as R (then (e, p) follow
from lambda_i ~ R_i^-2, the convention of pm3d.zeldovich_axes, pm3d.py:20-23) or as (e, p)
with R_i = R_bar A_i(e, p).
"""
from __future__ import annotations

import functools
import math
from dataclasses import dataclass, field

import numpy as np

DELTA_C = 1.686
A_START_CFG = 0.01
R_CONFIG1 = (0.10, 0.09, 0.08)
R_BAR = float(np.cbrt(np.prod(R_CONFIG1)))   # 0.0896...: geometric mean of the config-1 radii


def zeldovich_axes(e: float, p: float) -> np.ndarray:
    lam = np.array([1.0 + 3.0 * e + p, 1.0 - 2.0 * p, 1.0 - 3.0 * e + p]) / 3.0
    ax = lam ** -0.5
    return ax / np.prod(ax) ** (1.0 / 3.0)


def implied_ep(R) -> tuple[float, float]:
    """(e, p) of axes R under lambda_i ~ R_i^-2 normalised to sum lambda = 1."""
    lam = np.sort(np.asarray(R, dtype=np.float64) ** -2.0)[::-1]
    lam = lam / lam.sum()
    return float((lam[0] - lam[2]) / 2.0), float((lam[0] + lam[2] - 2.0 * lam[1]) / 2.0)


def _shape_coeffs(R):
    """b_i = (2/3) R1 R2 R3 R_D(R_j^2, R_k^2, R_i^2) - 2/3 (Carlson's R_D)."""
    from scipy.special import elliprd
    x = np.asarray(R) ** 2
    pr = float(np.prod(R))
    return np.array([2.0 / 3.0 * pr * elliprd(x[1], x[2], x[0]),
                     2.0 / 3.0 * pr * elliprd(x[0], x[2], x[1]),
                     2.0 / 3.0 * pr * elliprd(x[0], x[1], x[2])]) - 2.0 / 3.0


def collapse_times(e: float, p: float, delta_i: float = 1e-2, f_freeze: float = 0.01,
                   max_step: float = 50.0) -> np.ndarray:
    """Bond & Myers (1996) collapse times t1 <= t2 <= t3 (units of t_i; EdS, G = 1) of the three
    axes of a homogeneous ellipsoid with Zel'dovich eigenvalues delta_i (1+3e+p, 1-2p, 1-3e+p)/3
    and the external tide in linear theory: the model of pbhgr/scripts/ellipsoidal_collapse.py:
    14-54, pinned against it by tests/golden/collapse_times.npz.

    The axes obey R_i'' = -4 pi rho_b R_i [(1 + delta)/3 + b_i delta/2 + (lambda_i - delta_i/3) a]
    with a = t^(2/3), rho_b = 1/(6 pi t^2), delta = a^3/(R1 R2 R3) - 1 and the interior shape
    coefficients b_i (Carlson's R_D).  The run is integrated in segments, one per freeze: an
    axis freezes (its size held, its velocity zeroed) when it falls to f_freeze of its largest
    size as known at the start of the segment, and the largest sizes are updated from the state
    at the end of each segment.  max_step bounds the integrator's step; the reference bounds it
    by 0.02 t_segment, which changes the times by less than 1e-6 relative (the fixture test)."""
    from scipy.integrate import solve_ivp
    lam = delta_i * np.array([1 + 3 * e + p, 1 - 2 * p, 1 - 3 * e + p]) / 3.0
    frozen = np.zeros(3, dtype=bool)
    r_hold = np.zeros(3)
    t_col = np.full(3, np.nan)
    r_top = 1.0 - lam
    t, y = 1.0, np.concatenate([1.0 - lam, (2.0 / 3.0) * (1.0 - 2.0 * lam)])
    t_end = 1e5

    def rhs(tt, yy):
        R = np.where(frozen, r_hold, np.maximum(yy[:3], 1e-9))
        a = tt ** (2.0 / 3.0)
        rho_b = 1.0 / (6.0 * math.pi * tt * tt)
        delta = a ** 3 / np.prod(R) - 1.0
        acc = -4.0 * math.pi * rho_b * R * ((1.0 + delta) / 3.0 + 0.5 * _shape_coeffs(R) * delta
                                           + (lam - delta_i / 3.0) * a)
        return np.concatenate([np.where(frozen, 0.0, yy[3:]), np.where(frozen, 0.0, acc)])

    while t < t_end and not frozen.all():
        floor = f_freeze * r_top.copy()
        live = np.flatnonzero(~frozen)

        def hit(tt, yy, live=live, floor=floor):
            return float(np.min(yy[live] - floor[live]))
        hit.terminal = True
        hit.direction = -1
        sol = solve_ivp(rhs, (t, t_end), y, events=hit, rtol=1e-8, atol=1e-12, method="DOP853",
                        max_step=max_step)
        t, y = float(sol.t[-1]), sol.y[:, -1].copy()
        r_top = np.maximum(r_top, y[:3])
        if sol.status != 1:
            break
        gap = np.where(frozen, np.inf, y[:3] - f_freeze * r_top)
        i = int(np.argmin(gap))
        frozen[i] = True
        r_hold[i] = y[i]
        t_col[i] = t
    return t_col


@functools.lru_cache(maxsize=4096)
def _first_axis_time(e: float, p: float) -> float:
    return float(collapse_times(e, p)[0])


def first_axis_ratio(e: float, p: float) -> float:
    """t1/t_sph for Zel'dovich ellipticity e and prolateness p (rounded to 1e-4 for caching):
    the first axis's collapse time over the spherical (e = p = 0) one."""
    e, p = round(float(e), 4), round(float(p), 4)
    return _first_axis_time(e, p) / _first_axis_time(0.0, 0.0)


def delta0_for_collapse(a_collapse_cfg: float, e: float, p: float) -> float:
    """Initial central overdensity (at a_cfg = 0.01) whose first axis collapses at a_collapse_cfg."""
    a_c_pm = a_collapse_cfg / A_START_CFG
    return DELTA_C * first_axis_ratio(e, p) ** (2.0 / 3.0) / a_c_pm


@dataclass
class PeakSpec:
    N: int
    R: tuple
    delta0: float
    seed: int
    L: float = 1.0
    noise_frac: float = 0.01
    e: float = 0.0
    p: float = 0.0
    a_collapse_cfg: float = 0.8
    steps: int = 100
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.N ** 3

    def ratio(self) -> float:
        """Step ratio of `steps` steps uniform in ln a over a factor 100 (a_cfg 0.01 -> 1)."""
        return 100.0 ** (1.0 / self.steps) - 1.0


def single_peak(N: int = 32, steps: int = 100, seed: int = 0) -> PeakSpec:
    """The plain-run recipe: R = (0.10, 0.09, 0.08) L, first axis collapsing at a_cfg = 0.8."""
    e, p = implied_ep(R_CONFIG1)
    return PeakSpec(N=N, R=R_CONFIG1, delta0=delta0_for_collapse(0.8, e, p), seed=seed, e=e, p=p,
                    a_collapse_cfg=0.8, steps=steps, meta={"rule": "delta0 = 1.686 (t1/t_sph)^(2/3)/80"})


def large_peak(N: int = 512, steps: int = 300, seed: int = 0) -> PeakSpec:
    """e = 0.3, p = 0.1, axes R_bar A_i(e, p), first axis collapsing at a_cfg = 0.5."""
    e, p = 0.3, 0.1
    R = tuple(float(v) for v in R_BAR * zeldovich_axes(e, p))
    return PeakSpec(N=N, R=R, delta0=delta0_for_collapse(0.5, e, p), seed=seed, e=e, p=p, a_collapse_cfg=0.5,
                    steps=steps)


def ensemble(npeaks: int = 64, sizes=(32, 64, 128, 256), steps: int = 150, seed: int = 1234,
             e_range=(0.0, 0.3), p_range=(-0.1, 0.1), a_range=(0.3, 1.0)) -> list[PeakSpec]:
    """Mixed-size ensemble: mesh uniform over `sizes`, e ~ U(e_range), p ~ U(p_range), collapse
    a_cfg log-uniform over a_range, peak i seeded with seed + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(npeaks):
        N = int(rng.choice(sizes))
        e = float(rng.uniform(*e_range))
        p = float(rng.uniform(*p_range))
        a_c = float(np.exp(rng.uniform(np.log(a_range[0]), np.log(a_range[1]))))
        R = tuple(float(v) for v in R_BAR * zeldovich_axes(e, p))
        out.append(PeakSpec(N=N, R=R, delta0=delta0_for_collapse(a_c, e, p), seed=seed + i, e=e, p=p,
                            a_collapse_cfg=a_c, steps=steps))
    return out
