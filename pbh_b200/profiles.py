"""Curvature-profile tables for `PM3D.make_ic` and the LTB units of the pm3d driver (host side).

`PM3D.make_ic(mu, profile_spline, ...)` takes the normalised curvature profile Psi(r) as a
spline (pbhgr/pbhgr/pm3d.py:40-52); the reference builds it with `profile_table(name)`
(pbhgr/pbhgr/profiles.py:50-62) and the driver scales its box and run time with the growing-
mode LTB solution of that profile (pbhgr/scripts/pm3d_peak.py:16-19, pbhgr/pbhgr/ltb.py).
This module provides both, so a run can be set up without the reference package:

* profile_table('yoo')     Psi = exp(-r^2/6)                         (profiles.py:52-53)
* profile_table('ln<D>')   mean BBKS peak profile of a log-normal spectrum of width D
                           (profiles.py:22-41)
* profile_table('tophat')  super-Gaussian exp(-(r/2.5)^4)            (profiles.py:43-47)
* ltb_units(mu, name, table) -> (r_m, t_H, t_C(0))                   (ltb.py:16-23, 26-35, 104-114)

The tables use the reference's radius grid and quadrature (same grids, same rectangle rule),
so the splines agree to rounding.
"""
from __future__ import annotations

import numpy as np
from scipy.interpolate import CubicSpline

H_I = 5.0
T_I = 2.0 / (3.0 * H_I)


def _bbks_theta(gamma: float, gnu: float) -> float:
    """theta(gamma, gamma nu) of BBKS (1986) eq. 6.14: the mean curvature of a peak of height nu
    is x_bar = gamma nu + theta."""
    num = 3.0 * (1.0 - gamma ** 2) + (1.216 - 0.9 * gamma ** 4) * np.exp(-(gamma / 2.0) * (gnu / 2.0) ** 2)
    den = np.sqrt(3.0 * (1.0 - gamma ** 2) + 0.45 + (gnu / 2.0) ** 2) + gnu / 2.0
    return num / den


def lognormal_peak_profile(width: float, nu: float = 4.0, r_max: float = 40.0, n_r: int = 4001) -> dict:
    """Mean profile of a peak of height nu (in units of sigma_0) of a Gaussian field whose
    dimensionless power is log-normal, P(k) = exp(-ln^2 k / (2 width^2)) with k in units of the
    spectral peak.  Conditional mean of the field given its value and Laplacian at the peak:
    F(r) = s0^2 [psi(r), lap psi(r)] C^-1 [nu s0, -x_bar s2], C = [[s0^2, -s1^2], [-s1^2, s2^2]],
    normalised to F(0) = 1 (profiles.py:22-41)."""
    lnk = np.linspace(-8.0 * width - 2.0, 8.0 * width + 2.0, 20001)
    dlnk = lnk[1] - lnk[0]
    k = np.exp(lnk)
    P = np.exp(-lnk ** 2 / (2.0 * width ** 2))
    s0 = np.sqrt(P.sum() * dlnk)
    s1 = np.sqrt((P * k ** 2).sum() * dlnk)
    s2 = np.sqrt((P * k ** 4).sum() * dlnk)
    gamma = s1 ** 2 / (s0 * s2)
    r = np.linspace(0.0, r_max, n_r)
    psi = np.empty(n_r)
    lap = np.empty(n_r)
    for lo in range(0, n_r, 200):              # blocks of radii keep the kr table small
        kr = np.outer(r[lo:lo + 200], k)
        j0 = np.where(kr > 1e-8, np.sin(kr) / np.maximum(kr, 1e-300), 1.0)
        psi[lo:lo + 200] = (j0 @ P) * dlnk / s0 ** 2
        lap[lo:lo + 200] = -((j0 * k[None, :] ** 2) @ P) * dlnk / s0 ** 2
    x_bar = gamma * nu + _bbks_theta(gamma, gamma * nu)
    C = np.array([[s0 ** 2, -s1 ** 2], [-s1 ** 2, s2 ** 2]])
    w = np.linalg.solve(C, np.array([nu * s0, -x_bar * s2]))
    F = s0 ** 2 * (psi * w[0] + lap * w[1])
    return dict(r=r, Psi=F / F[0], psi=psi, gamma=gamma, R_star=np.sqrt(3.0) * s1 / s2, x_bar=x_bar, nu=nu,
                Delta=width, s0=s0)


def tophat_profile(r0: float = 2.5, n: float = 4.0, r_max: float = 40.0, n_r: int = 4001) -> dict:
    """Flat core with a steep edge: Psi = exp(-(r/r0)^n) (profiles.py:43-47)."""
    r = np.linspace(0.0, r_max, n_r)
    return dict(r=r, Psi=np.exp(-(r / r0) ** n), r0=r0, n=n)


def profile_table(name: str) -> dict:
    """'yoo' | 'ln<width>' | 'tophat' -> dict with r, Psi and the clamped cubic spline of Psi."""
    if name == "yoo":
        r = np.linspace(0.0, 40.0, 4001)
        d = dict(r=r, Psi=np.exp(-r ** 2 / 6.0))
    elif name.startswith("ln"):
        d = lognormal_peak_profile(float(name[2:]))
    elif name == "tophat":
        d = tophat_profile()
    else:
        raise ValueError(f"unknown profile {name!r}")
    d["spline"] = CubicSpline(d["r"], d["Psi"], bc_type=((1, 0.0), (1, 0.0)))
    return d


def ltb_units(mu: float, name: str = "yoo", table: dict | None = None, k: float = 1.0, h_i: float = H_I):
    """(r_m, t_H, t_C(0)) of the growing-mode LTB solution of the profile zeta = mu Psi(k r):
    Misner-Sharp mass m = (H_i^2/2)(e^zeta r)^3, energy E = r zeta' (1 + r zeta'/2), collapse time
    t_C(r) = 2 pi m / (-2E)^(3/2).  The Yoo Gaussian has r_m = sqrt(6)/k and
    t_H = t_i (sqrt(6) H_i / k)^3; a tabulated profile takes r_m at the maximum of -E and
    t_H = t_i (r_m H_i)^3.  t_C(0) is the limit at r -> 0 (taken at r = 1e-6), or t_C(r_m) where
    that limit is not finite (ltb.py:16-35, 104-114; pm3d_peak.py:16-19)."""
    t_i = 2.0 / (3.0 * h_i)
    if name == "yoo":
        zeta = lambda r: mu * np.exp(-k ** 2 * r ** 2 / 6.0)
        dzeta = lambda r: -(k ** 2 * r / 3.0) * zeta(r)
        r_m = np.sqrt(6.0) / k
        t_h = t_i * (np.sqrt(6.0) * h_i / k) ** 3
    else:
        table = table or profile_table(name)
        s, s1 = table["spline"], table["spline"].derivative(1)
        zeta = lambda r: mu * s(np.asarray(r, dtype=float) * k)
        dzeta = lambda r: mu * k * s1(np.asarray(r, dtype=float) * k)
        energy = lambda r: r * dzeta(r) * (1.0 + 0.5 * r * dzeta(r))
        grid = np.linspace(1e-3, table["r"][-1] * 0.9, 20000)
        r_m = float(grid[np.argmax(-energy(grid))])
        t_h = t_i * (r_m * h_i) ** 3

    def t_c(r):
        mass = 0.5 * h_i ** 2 * (np.exp(zeta(r)) * r) ** 3
        rz = r * dzeta(r)
        e = rz * (1.0 + 0.5 * rz)
        with np.errstate(invalid="ignore"):
            return float(2.0 * np.pi * mass / (-2.0 * e) ** 1.5)

    tc0 = t_c(1e-6)
    if not np.isfinite(tc0):
        tc0 = t_c(r_m)
    return float(r_m), float(t_h), tc0
