"""Newtonian 3D PM run of one triaxial peak on the B200 engine: the command-line driver of
pbhgr/scripts/pm3d_peak.py with the same arguments, console lines and JSON output, so runs
can be compared file for file.

    python -m pbh_b200.pm3d_peak --mu 0.1 --e 0 --p 0 --N 128 --Np 64 --L 8 --tend 40 \\
        [--tail 0.05 --k1 2 --k2 10] [--profile yoo] [--out runs/pm3d]

The loop is the reference's (pm3d_peak.py:24-33): da = min(da_frac a, a_end - a) until
a_end = (tend t_H / t_i)^(2/3), `analyse` every max(0.5, 0.02 t_C(0)/t_H) in t/t_H and at the
end.  Here the steps run on the device (one graph replay each, the schedule in device memory)
and the host only looks in at the diagnostic times; max delta comes from the device's own
deposit statistics instead of a copy of the density grid.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from .pm3d import PM3D, T_I, analyse
from .profiles import ltb_units, profile_table


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--mu", type=float, default=0.1)
    ap.add_argument("--e", type=float, default=0.0)
    ap.add_argument("--p", type=float, default=0.0)
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--Np", type=int, default=64)
    ap.add_argument("--L", type=float, default=8.0)
    ap.add_argument("--tend", type=float, default=40.0)
    ap.add_argument("--tail", type=float, default=0.0)
    ap.add_argument("--k1", type=float, default=2.0)
    ap.add_argument("--k2", type=float, default=10.0)
    ap.add_argument("--profile", default="yoo")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--smooth", type=float, default=2.0)
    ap.add_argument("--da_frac", type=float, default=0.02)
    ap.add_argument("--out", default="runs/pm3d")
    return ap.parse_args(argv)


def tag_of(args) -> str:
    """Run name of pm3d_peak.py:21 (the JSON file is named after it)."""
    tag = f"mu{args.mu:g}_e{args.e:g}_p{args.p:g}_N{args.N}_Np{args.Np}_L{args.L:g}_sm{args.smooth:g}"
    if args.tail > 0:
        tag += f"_tail{args.tail:g}_k{args.k1:g}-{args.k2:g}_s{args.seed}"
    if args.profile != "yoo":
        tag += f"_{args.profile}"
    return tag


def main(argv=None) -> dict:
    args = parse(argv)
    Path(args.out).mkdir(parents=True, exist_ok=True)
    table = profile_table(args.profile)
    table["name"] = args.profile
    rm, t_h, tc0 = ltb_units(args.mu, args.profile, table)
    pm = PM3D(args.N, args.L * rm, args.Np, seed=args.seed, smooth=args.smooth).make_ic(
        args.mu, table["spline"], args.e, args.p, args.tail, (args.k1, args.k2))
    tag = tag_of(args)
    c = args.N // 2
    print(f"PM3D {tag}: box {args.L} r_m = {args.L * rm:.2f}/k, dx = {pm.dx:.4f}/k ({pm.dx / rm:.4f} r_m), "
          f"{args.Np ** 3} particles, m_part = {pm.m_part:.3e}; axes A = {np.round(pm.A, 3)}; "
          f"t_C(0) = {tc0 / t_h:.2f} t_H, run to {args.tend} t_H; central delta_lin(a=1) = "
          f"{pm.delta_lin[c, c, c]:.4f} (expected 0.4 mu/25 = {0.4 * args.mu / 25:.4f}); "
          f"tail rms on grid = {pm.tail_rms_grid:.4f}", flush=True)
    a_end = (args.tend * t_h / T_I) ** (2.0 / 3.0)
    rows = []
    t0 = time.time()
    state = {"next": 0.0}

    def diag(pm_, a, step):
        t = T_I * a ** 1.5
        if t / t_h < state["next"] and a < a_end:
            return
        d = analyse(pm_, a)
        dmax = pm_.delta_max()
        d.update(t=t, t_over_tH=t / t_h, t_over_tC0=t / tc0, step=step, delta_max=float(dmax))
        rows.append(d)
        print(f"step {step:5d} t/t_H={t / t_h:7.3f} (t/tC0={t / tc0:.3f}) a={a:8.2f} delta_max={dmax:8.1f} | "
              f"comoving axes(0.1/0.2/0.3 r_m)={np.round(d['axes_com_0.1'], 3)} {np.round(d['axes_com_0.2'], 3)} "
              f"{np.round(d['axes_com_0.3'], 3)} hoop(0.2)={d['hoop_0.2']:.4f} | m(<1,2,4,8 cells)="
              f"{d['m_in_1c']:.2f} {d['m_in_2c']:.2f} {d['m_in_4c']:.2f} {d['m_in_8c']:.2f} "
              f"C(<2c)={d['C_2c']:.4f} | {time.time() - t0:.0f}s", flush=True)
        state["next"] = t / t_h + max(0.5, 0.02 * tc0 / t_h)

    pm.run(a_end, args.da_frac, a=1.0, callback=diag, every=1)
    result = dict(args=vars(args), rows=rows, rm=rm, t_H=t_h, tC0=tc0, dx=pm.dx, m_part=pm.m_part)
    with open(Path(args.out) / f"{tag}.json", "w") as f:
        json.dump(result, f)
    print("done", f"{time.time() - t0:.0f}s")
    return result


if __name__ == "__main__":
    main()
