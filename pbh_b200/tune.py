"""Autotuner for the per-peak super-tile side.

The super-tile (TS^3 cells) is the unit of the push, the deposit and the particle grouping.
Larger tiles amortise the force-patch staging and the deposit's node phases over more
particles; smaller tiles give more CTAs, which matters for a small mesh run alone.  The tuner
times a few graph-replayed steps of a recipe peak for each candidate side on the current GPU
and keeps the fastest per mesh size.  Results are cached in a JSON file next to this module,
keyed by the GPU, the library build and the mesh size, so a size is tuned once per build.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

from . import _lib

CACHE = Path(__file__).resolve().parent / "_tune_cache.json"
CANDIDATES = (4, 8, 16)


def _key(N: int, device: int) -> str:
    torch = _lib.require_cuda()
    props = torch.cuda.get_device_properties(device)
    so = Path(_lib.LIB_PATH)
    st = so.stat()
    return f"{props.name}|sm{props.multi_processor_count}|lib{st.st_size}-{int(st.st_mtime)}|N{N}"


def _load_cache() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def _time_tile(N: int, tile: int, device: int, steps: int, warmup: int) -> float:
    """Device seconds per step of one recipe peak of mesh N with super-tile side `tile`."""
    torch = _lib.require_cuda()
    from . import recipe
    from .engine import Engine, PeakConfig
    from .ic import recipe_particles
    spec = recipe.single_peak(N=N, steps=steps + warmup + 4, seed=7)
    eng = Engine([PeakConfig(N=N, Np=N, L=spec.L, tile=tile)], device=device)
    try:
        x, p = recipe_particles(spec, device=device, device_noise=True)
        eng.set_particles(0, x, p, 1.0, mode=_lib.SCHED_RATIO, param=spec.ratio(), max_steps=spec.steps)
        del x, p
        eng.run(1 + warmup)
        stream = torch.cuda.ExternalStream(_lib.load().pm_engine_stream(eng._h), device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eng.sync()
        e0.record(stream)
        eng.run(steps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3 / steps
    finally:
        eng.close()


def autotune(sizes, device: int = 0, steps: int = 8, warmup: int = 3, use_cache: bool = True) -> dict:
    """{N: best super-tile side} for every mesh size in `sizes` (timed on `device`)."""
    cache = _load_cache() if use_cache else {}
    out, dirty = {}, False
    for N in sorted({int(n) for n in sizes}):
        key = _key(N, device)
        if key in cache:
            out[N] = int(cache[key]["tile"])
            continue
        cands = [t for t in CANDIDATES if t <= N]
        times = {t: _time_tile(N, t, device, steps, warmup) for t in cands}
        best = min(times, key=times.get)
        cache[key] = {"tile": best, "step_s": {str(t): v for t, v in times.items()}}
        out[N] = best
        dirty = True
    if dirty and use_cache:
        tmp = CACHE.with_suffix(f".{os.getpid()}.tmp")  # one writer per process (ranks share the file)
        tmp.write_text(json.dumps(cache, indent=1))
        os.replace(tmp, CACHE)
    return out


def tuned_times(N: int, device: int = 0) -> dict:
    """The cached per-candidate step times of mesh N (empty if not tuned)."""
    return _load_cache().get(_key(N, device), {}).get("step_s", {})
