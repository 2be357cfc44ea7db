"""Python handle over the native engine (libpmb200.so, include/pmb200.h).

An ``Engine`` holds one or more independent peaks (one PM3D run each) resident on one GPU:
particle state, meshes, cuFFT plans and the captured step graph.  Inputs and outputs are
torch CUDA tensors; the engine runs on its own stream and every call that hands data back
synchronizes it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

GRADIENTS = {"spectral": 0, "fd2": 1, "fd4": 2}


@dataclass
class PeakConfig:
    N: int
    Np: int
    L: float
    smooth: float = 0.0
    tile: int = 0
    gradient: str = "spectral"
    n: int = 0          # explicit particle count (0: Np**3)

    def cstruct(self) -> _lib.PeakCfg:
        return _lib.PeakCfg(int(self.N), int(self.Np), int(self.tile), GRADIENTS[self.gradient],
                            float(self.L), float(self.smooth), int(self.n))

    @property
    def n_particles(self) -> int:
        return int(self.n) if self.n else int(self.Np) ** 3


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def engine_flags(graph: bool = True, full_every: int = 0, dynamic: bool = False, bucket_sort: bool = True,
                 native_fft: bool = True, tight_bins: bool = False) -> int:
    """The `flags` word of pm_engine_create: bits 8..15 the super-tile re-sort period (0: never;
    bucket_sort=False: every step; periods above 255 become 255), bit 1 graph replay, bit 2
    served (dynamic) mode, bit 3 the native transforms, bit 16 bins without spare capacity."""
    every = int(full_every) if bucket_sort else 1
    return ((max(0, min(every, 255)) & 0xFF) << 8) | (_lib.FLAG_GRAPH if graph else 0) | \
        (_lib.FLAG_DYNAMIC if dynamic else 0) | (_lib.FLAG_NATIVE_FFT if native_fft else 0) | \
        (_lib.FLAG_TIGHT_BINS if tight_bins else 0)


class Engine:
    def __init__(self, peaks, device: int = 0, graph: bool = True, full_every: int = 0, dynamic: bool = False,
                 bucket_sort: bool = True, native_fft: bool = True, tight_bins: bool = False):
        torch = _lib.require_cuda()
        self._torch = torch
        lib = _lib.load()
        self._lib = lib
        self.cfgs = [p if isinstance(p, PeakConfig) else PeakConfig(**p) for p in peaks]
        arr = (_lib.PeakCfg * len(self.cfgs))(*[c.cstruct() for c in self.cfgs])
        h = C.c_void_p()
        self.device = int(device)
        # The push appends every particle to the bin of its new super-tile; every `full_every`
        # steps (0: never, the default) each super-tile is re-sorted by cell (bucket_sort=False:
        # every step).  Results do not depend on the choice: the deposit is order-independent bit
        # for bit.  tight_bins:
        # bins without spare capacity, so that almost every step overflows and relayouts (a test
        # of that path; same results).
        # dynamic: served runs; no graph, and each step's FFTs cover only the slots in use.
        # native_fft: 64^3-512^3 meshes use the native transform with the Green multiply fused
        # (False: cuFFT and the separate Green kernel, as for every other mesh size).
        flags = engine_flags(graph, full_every, dynamic, bucket_sort, native_fft, tight_bins)
        self.npeaks = len(self.cfgs)
        torch.cuda.set_device(self.device)
        check(lib.pm_engine_create(arr, len(self.cfgs), self.device, flags, C.byref(h)), "pm_engine_create")
        self._h = h

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.pm_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(self._lib.pm_engine_device_bytes(self._h))

    def sync(self):
        check(self._lib.pm_engine_sync(self._h), "pm_engine_sync")

    def _dev(self, a, dtype):
        torch = self._torch
        t = torch.as_tensor(a, dtype=dtype, device=f"cuda:{self.device}").contiguous()
        torch.cuda.current_stream(self.device).synchronize()
        return t

    # ------------------------------------------------------------------ state
    def set_particles(self, peak: int, x, p, a0: float, mode: int = _lib.SCHED_EXPLICIT, param: float = 0.0,
                      a_end: float = 0.0, max_steps: int = 0):
        torch = self._torch
        n = self.cfgs[peak].n_particles
        xt = self._dev(x, torch.float64).reshape(n, 3)
        pt = self._dev(p, torch.float64).reshape(n, 3)
        check(self._lib.pm_set_particles(self._h, peak, _ptr(xt), _ptr(pt), float(a0), int(mode), float(param),
                                         float(a_end), int(max_steps)), "pm_set_particles")

    def run(self, nsteps: int):
        check(self._lib.pm_run(self._h, int(nsteps)), "pm_run")

    def step_explicit(self, peak: int, a: float, da: float):
        check(self._lib.pm_step_explicit(self._h, peak, float(a), float(da)), "pm_step_explicit")

    def particles(self, peak: int):
        torch = self._torch
        n = self.cfgs[peak].n_particles
        x = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{self.device}")
        p = torch.empty_like(x)
        torch.cuda.current_stream(self.device).synchronize()
        check(self._lib.pm_get_particles(self._h, peak, _ptr(x), _ptr(p)), "pm_get_particles")
        return x, p

    def acc(self, peak: int, a: float):
        torch = self._torch
        n = self.cfgs[peak].n_particles
        out = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{self.device}")
        torch.cuda.current_stream(self.device).synchronize()
        check(self._lib.pm_get_acc(self._h, peak, float(a), _ptr(out)), "pm_get_acc")
        return out

    def delta(self, peak: int):
        torch = self._torch
        N = self.cfgs[peak].N
        out = torch.empty((N, N, N), dtype=torch.float32, device=f"cuda:{self.device}")
        torch.cuda.current_stream(self.device).synchronize()
        check(self._lib.pm_get_delta(self._h, peak, _ptr(out)), "pm_get_delta")
        return out

    def counts(self, peak: int):
        torch = self._torch
        N = self.cfgs[peak].N
        out = torch.empty((N, N, N), dtype=torch.float64, device=f"cuda:{self.device}")
        torch.cuda.current_stream(self.device).synchronize()
        check(self._lib.pm_get_counts(self._h, peak, _ptr(out)), "pm_get_counts")
        return out

    def release(self, peak: int):
        check(self._lib.pm_release(self._h, peak), "pm_release")

    def clock(self, peak: int) -> _lib.ClockInfo:
        c = _lib.ClockInfo()
        check(self._lib.pm_get_clock(self._h, peak, C.byref(c)), "pm_get_clock")
        return c

    def stats(self, peak: int) -> _lib.StatsInfo:
        s = _lib.StatsInfo()
        rc = self._lib.pm_get_stats(self._h, peak, C.byref(s))
        check(rc, "pm_get_stats")
        return s


def interp64(F, X, L: float):
    """PM3D.interp on the GPU in float64 (pm3d.py:91-99)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    Ft = torch.as_tensor(np.asarray(F, dtype=np.float64)).cuda().contiguous()
    Xt = torch.as_tensor(np.asarray(X, dtype=np.float64)).cuda().contiguous()
    out = torch.empty(Xt.shape[0], dtype=torch.float64, device="cuda")
    if Xt.shape[0] == 0:        # no positions: an empty gather, as the reference's indexing gives
        return out
    torch.cuda.synchronize()
    check(lib.pm_interp64(_ptr(Ft), _ptr(Xt), Xt.shape[0], Ft.shape[0], float(L), _ptr(out)), "pm_interp64")
    return out


def deposit64(X, N: int, L: float):
    """PM3D.deposit on the GPU (pm3d.py:81-89): float64 CIC counts of arbitrary positions, from
    64-bit fixed-point integer sums (independent of the order of X)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    Xt = torch.as_tensor(np.asarray(X, dtype=np.float64).reshape(-1, 3)).cuda().contiguous()
    if Xt.shape[0] == 0:        # no particles: zero counts, as the reference's bincount gives
        return torch.zeros((N, N, N), dtype=torch.float64, device="cuda")
    work = torch.empty(N ** 3, dtype=torch.int64, device="cuda")
    out = torch.empty((N, N, N), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    check(lib.pm_deposit64(_ptr(Xt), Xt.shape[0], int(N), float(L), _ptr(work), _ptr(out)), "pm_deposit64")
    return out


def sort_u64(keys, lo: int = 0, hi: int = 64):
    """Stable radix sort of uint64 keys over bits [lo, hi) on the GPU: (sorted keys, permutation)."""
    torch = _lib.require_cuda()
    lib = _lib.load()
    k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
    kin = torch.from_numpy(k.view(np.int64)).cuda()
    n = kin.numel()
    kout = torch.empty_like(kin)
    tk = torch.empty_like(kin)
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    tv = torch.empty_like(perm)
    torch.cuda.synchronize()
    rc = lib.pm_sort_u64(_ptr(kin), _ptr(kout), _ptr(perm), _ptr(tk), _ptr(tv), n, int(lo), int(hi))
    check(rc, "pm_sort_u64")
    if rc:
        raise _lib.PMError("pm_sort_u64: a bounded look-back wait gave up")
    return kout.cpu().numpy().view(np.uint64), perm.cpu().numpy().view(np.uint32)
