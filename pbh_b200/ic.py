"""Initial particles on the GPU (float64): PM3D.make_ic (pbhgr/pbhgr/pm3d.py:40-73) and the
benchmark's Gaussian-peak recipe, through pm_make_ic of libpmb200.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

KIND_ZETA, KIND_GAUSS = 0, 1


def make_particles(N: int, Np: int, L: float, kind: int, amp: float, axes, *, spline=None, noise=None,
                   tail_rms: float = 0.0, tail_k=(2.0, 10.0), noise_frac: float = 0.0, device: int = 0,
                   delta_lin: bool = False, noise_seed: int = 0):
    """Returns (x, p, delta_lin or None, noise_rms): x, p are (Np^3, 3) float64 CUDA tensors in
    lattice order.  `noise` (N^3 standard normals) may be a numpy array, a pinned CPU tensor or
    a CUDA tensor; without it, a nonzero `noise_seed` draws the normals on the device."""
    torch = _lib.require_cuda()
    dev = f"cuda:{device}"
    n = Np ** 3
    x = torch.empty((n, 3), dtype=torch.float64, device=dev)
    p = torch.empty_like(x)
    dl = torch.empty((N, N, N), dtype=torch.float64, device=dev) if delta_lin else None
    prm = _lib.ICParams()
    prm.N, prm.Np, prm.L, prm.kind, prm.amp = int(N), int(Np), float(L), int(kind), float(amp)
    prm.axes = (C.c_double * 3)(*[float(v) for v in axes])
    keep = []
    if spline is not None:
        xs = np.ascontiguousarray(spline.x, dtype=np.float64)
        cs = np.ascontiguousarray(spline.c, dtype=np.float64)
        if cs.ndim != 2 or cs.shape[0] != 4:
            raise ValueError("profile_spline must be a cubic piecewise polynomial (scipy CubicSpline)")
        keep += [xs, cs]
        prm.spline_x = xs.ctypes.data_as(C.c_void_p)
        prm.spline_c = cs.ctypes.data_as(C.c_void_p)
        prm.spline_m = cs.shape[1]
    nt = None
    if noise is not None:
        nt = torch.as_tensor(noise, dtype=torch.float64).to(dev, non_blocking=True).contiguous()
        prm.noise = nt.data_ptr()
    prm.tail_rms, prm.k1, prm.k2 = float(tail_rms), float(tail_k[0]), float(tail_k[1])
    prm.noise_frac = float(noise_frac)
    prm.noise_seed = int(noise_seed) if noise is None else 0
    rms = C.c_double(0.0)
    torch.cuda.synchronize(dev)
    with torch.cuda.device(dev):
        check(_lib.load().pm_make_ic(C.byref(prm), x.data_ptr(), p.data_ptr(), 0 if dl is None else dl.data_ptr(),
                                     C.byref(rms)), "pm_make_ic")
    return x, p, dl, float(rms.value)


def recipe_particles(spec, device: int = 0, noise=None, device_noise: bool = False):
    """Particles of a recipe PeakSpec (pbh_b200.recipe).  Noise defaults to the peak's own
    generator default_rng(seed).standard_normal((N, N, N)) (numpy's stream, as the reference
    draws it); device_noise draws it on the GPU from the seed instead."""
    if noise is None and spec.noise_frac > 0 and not device_noise:
        noise = np.random.default_rng(spec.seed).standard_normal((spec.N,) * 3)
    x, p, _, _ = make_particles(spec.N, spec.N, spec.L, KIND_GAUSS, spec.delta0, spec.R, noise=noise,
                                noise_frac=spec.noise_frac, device=device,
                                noise_seed=(spec.seed + 1) if device_noise else 0)
    return x, p
