"""ctypes binding of libpmb200.so (the C ABI declared in include/pmb200.h).

The library is built in-tree by ``pbh_b200/build.py``.  There is no fallback: if the
library or a CUDA device is missing, the product path raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpmb200.so"

SCHED_RATIO, SCHED_FRAC, SCHED_EXPLICIT = 0, 1, 2
STATE_IDLE, STATE_PRIME, STATE_RUN, STATE_FINALIZE, STATE_HOLD = 0, 1, 2, 3, 4
FLAG_BUCKET_SORT = 1
FLAG_GRAPH = 2
FLAG_DYNAMIC = 4
FLAG_NATIVE_FFT = 8
FLAG_TIGHT_BINS = 1 << 16
NOALLOC_MAX_KEYS = 1 << 18          # PM_NOALLOC_MAX_KEYS of include/pmb200.h


class PeakCfg(C.Structure):
    _fields_ = [("N", C.c_int), ("Np", C.c_int), ("tile", C.c_int), ("gradient", C.c_int),
                ("L", C.c_double), ("smooth", C.c_double), ("n", C.c_longlong)]


class ClockInfo(C.Structure):
    _fields_ = [("a", C.c_double), ("da", C.c_double), ("a_end", C.c_double), ("kpend", C.c_double),
                ("a_grid", C.c_double), ("mode", C.c_int), ("state", C.c_int), ("nsteps", C.c_int),
                ("max_steps", C.c_int), ("a_collapse", C.c_double)]


class StatsInfo(C.Structure):
    _fields_ = [("rho_max_over_mean", C.c_double), ("delta_max", C.c_double), ("mass_defect", C.c_double),
                ("status", C.c_uint), ("energy_samples", C.c_int), ("a_energy", C.c_double),
                ("momentum", C.c_double * 3), ("kinetic", C.c_double), ("potential", C.c_double),
                ("li_residual", C.c_double), ("li_scale", C.c_double), ("relayouts", C.c_int),
                ("relayouts_full", C.c_int)]


class ICParams(C.Structure):
    _fields_ = [("N", C.c_int), ("Np", C.c_int), ("L", C.c_double), ("kind", C.c_int), ("amp", C.c_double),
                ("axes", C.c_double * 3), ("spline_x", C.c_void_p), ("spline_c", C.c_void_p), ("spline_m", C.c_int),
                ("noise", C.c_void_p), ("tail_rms", C.c_double), ("k1", C.c_double), ("k2", C.c_double),
                ("noise_frac", C.c_double), ("noise_seed", C.c_ulonglong)]


# name -> (restype, argtypes)
_SIGS = {
    "pm_engine_create": (C.c_int, [C.POINTER(PeakCfg), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "pm_engine_destroy": (C.c_int, [C.c_void_p]),
    "pm_engine_sync": (C.c_int, [C.c_void_p]),
    "pm_engine_device_bytes": (C.c_longlong, [C.c_void_p]),
    "pm_set_particles": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_double,
                                   C.c_double, C.c_int]),
    "pm_run": (C.c_int, [C.c_void_p, C.c_int]),
    "pm_run_timed": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "pm_engine_stream": (C.c_void_p, [C.c_void_p]),
    "pm_engine_info": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pm_get_stats_all": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pm_get_clocks_all": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pm_step_explicit": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
    "pm_get_particles": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "pm_get_acc": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "pm_get_delta": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "pm_get_counts": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "pm_set_collapse_threshold": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int]),
    "pm_release": (C.c_int, [C.c_void_p, C.c_int]),
    "pm_load_peak": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_double,
                               C.c_double, C.c_int, C.c_double, C.c_int, C.c_void_p]),
    "pm_snapshot": (C.c_int, [C.c_void_p, C.c_int]),
    "pm_snapshot_read": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "pm_get_delta_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "pm_debug_sort_stall": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "pm_get_clock": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(ClockInfo)]),
    "pm_get_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(StatsInfo)]),
    "pm_make_ic": (C.c_int, [C.POINTER(ICParams), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    "pm_make_ic_async": (C.c_int, [C.POINTER(ICParams), C.c_void_p, C.c_void_p, C.c_void_p]),
    "pm_rell_keys": (C.c_int, [C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "pm_analyse_partials": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int, C.c_void_p]),
    "pm_ic_release_cache": (C.c_int, []),
    "pm_interp64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_double, C.c_void_p]),
    "pm_deposit64": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "pm_sort_u64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int,
                              C.c_int]),
    "pm_rfft3_native": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "pm_irfft3_native": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "pm_rfft3_256": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "pm_irfft3_256": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "pm_sort_u64_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_int,
                                      C.c_void_p]),
    "pm_cell_keys": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_void_p]),
}

_lib = None


class PMError(RuntimeError):
    pass


def load():
    """Load the library (once) and declare every entry point."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise PMError(f"{LIB_PATH} is missing: build it with `python pbh_b200/build.py`")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(rc: int, what: str) -> int:
    if rc < 0:
        if rc <= -2000:
            raise PMError(f"{what}: invalid argument (code {rc})")
        if rc <= -1000:
            raise PMError(f"{what}: cuFFT error {-1000 - rc}")
        raise PMError(f"{what}: CUDA error {-rc}")
    return rc


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise PMError("pbh_b200 needs a CUDA device (B200); none is visible")
    return torch
