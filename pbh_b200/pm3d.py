"""Drop-in replacement for ``pbhgr.pm3d`` (uniquehuman/pbh, pbhgr/pbhgr/pm3d.py) on one B200.

Same module surface: ``H_I, T_I, RHO_A3, zeldovich_axes, PM3D, analyse``; same constructor,
attributes, methods and return values.  Differences a caller can see:

* the particle state lives on the GPU as an int32 CIC cell + FP32 offset and FP32 momentum;
  ``x``/``p`` are reconstructed as float64 numpy arrays on access (lattice order);
* density, potential and forces are FP32 on the mesh; ``step``/``forces`` return float64
  numpy copies of them (or torch CUDA tensors with ``outputs="torch"``);
* ``analyse`` picks its 27/30 innermost Lagrangian particles with ties in r_ell_q broken by
  lattice index (the reference's default-kind argsort leaves tie order to numpy).

Every numerical step runs in the CUDA library ``libpmb200.so``; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .engine import Engine, PeakConfig, deposit64, interp64
from .ic import make_particles

H_I = 5.0                                   # pm3d.py:15-17
T_I = 2.0 / (3.0 * H_I)
RHO_A3 = 3.0 * H_I ** 2 / (8.0 * np.pi)


def zeldovich_axes(e: float, p: float):
    """Axis lengths A_i ~ lambda_i^(-1/2), prod A = 1 (pm3d.py:20-23)."""
    lam = np.array([1.0 + 3.0 * e + p, 1.0 - 2.0 * p, 1.0 - 3.0 * e + p]) / 3.0
    ax = lam ** -0.5
    return ax / np.prod(ax) ** (1.0 / 3.0)


class StateArray(np.ndarray):
    """Host copy of a PM3D's particle state (``pm.x`` or ``pm.p``), float64 in lattice order.

    The reference's ``x`` and ``p`` are plain arrays a caller may write into
    (pbhgr/pbhgr/pm3d.py:67-68); here the state lives on the GPU, so writing into this copy
    (item assignment, in-place arithmetic, ufuncs with ``out=``, through views too) marks it
    changed, and the owning PM3D loads it into the engine before its next device operation.
    A copy taken before the state changed on the device is stale, as an array the reference
    has rebound is: writing into it changes nothing."""

    def __array_finalize__(self, obj):
        # views share the state's memory and stay tied to it; a copy (own memory) is a plain
        # snapshot, as a copy of the reference's array is
        view = self.base is not None
        self._owner = getattr(obj, "_owner", None) if view else None
        self._gen = getattr(obj, "_gen", -1)

    def _touch(self):
        o = self._owner
        if o is not None and o._host_gen == self._gen:
            o._host_dirty = True

    def __setitem__(self, key, value):
        super().__setitem__(key, value)
        self._touch()

    def __array_ufunc__(self, ufunc, method, *inputs, out=None, **kwargs):
        args = [i.view(np.ndarray) if isinstance(i, StateArray) else i for i in inputs]
        if out is not None:
            for o in out:
                if isinstance(o, StateArray):
                    o._touch()
            kwargs["out"] = tuple(o.view(np.ndarray) if isinstance(o, StateArray) else o for o in out)
        res = getattr(ufunc, method)(*args, **kwargs)
        if out is not None:
            return out[0] if len(out) == 1 else out
        return res


def _lattice(Np: int, L: float) -> np.ndarray:
    q1 = (np.arange(Np) + 0.5) * (L / Np) - L / 2
    return np.stack(np.meshgrid(q1, q1, q1, indexing="ij"), axis=-1).reshape(-1, 3)


class PM3D:
    """Newtonian PM solver for one peak (pm3d.py:26-129), state resident on the GPU."""

    def __init__(self, N: int, L: float, Np: int, seed: int = 0, smooth: float = 0.0, *, device: int = 0,
                 tile: int = 0, gradient: str = "spectral", graph: bool = True, outputs: str = "numpy"):
        self.N, self.L, self.Np = int(N), float(L), int(Np)
        self.smooth = float(smooth)
        self.dx = self.L / self.N
        self.rng = np.random.default_rng(seed)
        self.m_part = RHO_A3 * self.L ** 3 / self.Np ** 3
        self.outputs = outputs
        self.device = int(device)
        self._cfg = PeakConfig(N=self.N, Np=self.Np, L=self.L, smooth=self.smooth, tile=tile, gradient=gradient)
        self._engine = Engine([self._cfg], device=device, graph=graph)
        self._torch = self._engine._torch
        self._kgrids = None
        self._loaded = False
        self.A = None
        self._delta_lin = None
        self.tail_rms_grid = 0.0
        self._host = None          # cached StateArray copies of x and p
        self._host_gen = 0
        self._host_dirty = False

    # ------------------------------------------------------------------ k-grids (pm3d.py:31-35)
    def _k(self):
        if self._kgrids is None:
            k1 = 2 * np.pi * np.fft.fftfreq(self.N, d=self.dx)
            kz = 2 * np.pi * np.fft.rfftfreq(self.N, d=self.dx)
            kx, ky, kzz = np.meshgrid(k1, k1, kz, indexing="ij")
            k2 = kx ** 2 + ky ** 2 + kzz ** 2
            k2[0, 0, 0] = 1.0
            self._kgrids = (kx, ky, kzz, k2)
        return self._kgrids

    kx = property(lambda self: self._k()[0])
    ky = property(lambda self: self._k()[1])
    kz = property(lambda self: self._k()[2])
    k2 = property(lambda self: self._k()[3])

    # ------------------------------------------------------------------ initial data
    def _ic(self, kind, amp, axes, spline=None, noise=None, tail_rms=0.0, tail_k=(2.0, 10.0), noise_frac=0.0):
        x, p, dl, rms = make_particles(self.N, self.Np, self.L, kind, amp, axes, spline=spline, noise=noise,
                                       tail_rms=tail_rms, tail_k=tail_k, noise_frac=noise_frac,
                                       device=self.device, delta_lin=True)
        self._engine.set_particles(0, x, p, 1.0)
        self._loaded = True
        self._stale()
        self._delta_lin = dl
        self._ic_xp = (x, p) if getattr(self, "keep_ic", False) else None
        self.A = np.asarray(axes, dtype=np.float64)
        return rms

    def make_ic(self, mu, profile_spline, e=0.0, p=0.0, tail_rms=0.0, tail_k=(2.0, 10.0)):
        """Zel'dovich particles of one triaxial peak (pm3d.py:40-73), computed on the GPU in float64."""
        A = zeldovich_axes(e, p)
        noise = self.rng.standard_normal((self.N,) * 3) if tail_rms > 0 else None   # pm3d.py:53
        rms = self._ic(0, mu, A, spline=profile_spline, noise=noise, tail_rms=tail_rms, tail_k=tail_k)
        self.tail_rms_grid = rms if tail_rms > 0 else 0.0
        self.A = A
        return self

    def make_peak(self, R, delta0: float, noise_frac: float = 0.01):
        """Gaussian linear density peak delta0 exp(-sum x_i^2/2R_i^2) plus noise with P(k) ~ k^-2
        at rms noise_frac*delta0, drawn from this run's generator, then the Zel'dovich tail of
        make_ic (pm3d.py:59-72).  A = R normalised to prod A = 1."""
        R = np.asarray(R, dtype=np.float64)
        noise = self.rng.standard_normal((self.N,) * 3) if noise_frac > 0 else None
        self.tail_rms_grid = self._ic(1, delta0, R, noise=noise, noise_frac=noise_frac)
        self.A = R / np.cbrt(np.prod(R))
        return self

    @property
    def q(self):
        return _lattice(self.Np, self.L)

    @property
    def delta_lin(self):
        return None if self._delta_lin is None else self._delta_lin.cpu().numpy()

    @property
    def r_ell_q(self):
        return np.sqrt(np.sum((self.q / self.A) ** 2, axis=1))

    # ------------------------------------------------------------------ particle state
    def _require(self):
        if not self._loaded:
            raise RuntimeError("no particles: call make_ic/make_peak or assign x and p first")

    def _prime(self):
        self._require()
        self._flush()
        if self._engine.clock(0).state == _lib.STATE_PRIME:
            self._engine.run(1)

    # Host copies of x and p: made on first access after the device state changed, loaded back
    # into the engine before the next device operation if they were written into.
    def _stale(self):
        self._host = None
        self._host_gen += 1
        self._host_dirty = False

    def _flush(self):
        if self._host is not None and self._host_dirty:
            x, p = self._host
            self._host_dirty = False
            self._assign(x=np.asarray(x), p=np.asarray(p))

    def _host_state(self):
        self._require()
        if self._host is None:
            xd, pd = self._engine.particles(0)
            arrs = []
            for t in (xd, pd):
                a = t.cpu().numpy().view(StateArray)
                a._owner, a._gen = self, self._host_gen
                arrs.append(a)
            self._host = tuple(arrs)
        return self._host

    @property
    def x(self):
        return self._host_state()[0]

    @x.setter
    def x(self, value):
        self._flush()
        self._assign(x=np.asarray(value, dtype=np.float64))

    @property
    def p(self):
        return self._host_state()[1]

    @p.setter
    def p(self, value):
        self._flush()
        self._assign(p=np.asarray(value, dtype=np.float64))

    def _assign(self, x=None, p=None):
        n = self.Np ** 3
        a0 = 1.0
        if self._loaded:
            cx, cp = self._engine.particles(0)
            a0 = self._engine.clock(0).a
        else:
            z = np.zeros((n, 3))
            cx, cp = z, z
        self._engine.set_particles(0, cx if x is None else x, cp if p is None else p, a0)
        self._loaded = True
        self._stale()

    @property
    def _acc_a(self):
        c = self._engine.clock(0)
        return c.a if c.state == _lib.STATE_HOLD and c.kpend != 0.0 else None

    @property
    def _acc(self):
        self._flush()
        a = self._acc_a
        return None if a is None else self._engine.acc(0, a).cpu().numpy()

    # ------------------------------------------------------------------ mesh operations
    def deposit(self, X):
        """CIC counts of arbitrary positions (pm3d.py:81-89): float64 on the GPU from 64-bit
        fixed-point integer sums (2^-39 of a particle per corner weight, order-independent)."""
        return deposit64(X, self.N, self.L).cpu().numpy()

    def interp(self, F, X):
        """CIC gather of mesh F at positions X (pm3d.py:91-99), float64 on the GPU."""
        return interp64(np.asarray(F, dtype=np.float64), np.asarray(X, dtype=np.float64).reshape(-1, 3),
                        self.L).cpu().numpy()

    def _out(self, t):
        """A device result as the reference returns it (float64 numpy), through a reused pinned
        staging buffer (one DMA instead of a pageable copy), or the device tensor itself."""
        if self.outputs == "torch":
            return t
        n = t.numel()
        pin = getattr(self, "_pin", None)
        if pin is None or pin.numel() < n or pin.dtype != t.dtype:
            pin = self._pin = self._torch.empty(n, dtype=t.dtype, pin_memory=True)
        pin[:n].copy_(t.reshape(-1))
        return pin[:n].numpy().reshape(tuple(t.shape)).astype(np.float64)

    def forces(self, a):
        """(-grad Phi at the particles, delta) for the current positions (pm3d.py:101-114)."""
        self._prime()
        return self._out(self._engine.acc(0, a)), self._out(self._engine.delta(0))

    # ------------------------------------------------------------------ leapfrog
    def step(self, a, da):
        """KDK step in a (pm3d.py:117-129); returns (a + da, delta at a + da)."""
        self._require()
        self._flush()
        self._engine.step_explicit(0, a, da)
        self._stale()
        return a + da, self._out(self._engine.delta(0))

    def close(self):
        """Release the device memory of this run now (it is also released with the object)."""
        self._engine.close()

    def delta_max(self) -> float:
        """Max delta of the latest deposit, from the device's own statistics (no grid copy)."""
        return float(self._engine.stats(0).delta_max)

    def energy(self) -> dict:
        """The engine's energy check at its last sample: total momentum, K, W and the
        Layzer-Irvine residual a(K + W) + int K da - a0 (K0 + W0) with its scale a(K + |W|)."""
        s = self._engine.stats(0)
        return dict(a=s.a_energy, samples=s.energy_samples, momentum=list(s.momentum), kinetic=s.kinetic,
                    potential=s.potential, layzer_irvine=s.li_residual, scale=s.li_scale)

    def run(self, a_end: float, da_frac: float = 0.02, a: float = 1.0, callback=None, every: int = 0):
        """The driver loop of pbhgr/scripts/pm3d_peak.py:24-33 on the device: da = min(da_frac a,
        a_end - a) until a_end, all steps replayed from one captured graph.  With ``callback``
        and ``every`` > 0 the loop pauses every ``every`` steps and calls callback(self, a, step)."""
        self._require()
        self._flush()
        eng = self._engine
        xd, pd = eng.particles(0)
        eng.set_particles(0, xd, pd, a, mode=_lib.SCHED_FRAC, param=da_frac, a_end=a_end)
        self._stale()
        eng.run(1)
        while True:
            c = eng.clock(0)
            if c.state in (_lib.STATE_IDLE, _lib.STATE_FINALIZE):
                break
            k = every if (callback and every > 0) else 64
            eng.run(k)
            c = eng.clock(0)
            if callback and every > 0:
                self._stale()
                callback(self, c.a, c.nsteps)
                self._flush()
        if eng.clock(0).state == _lib.STATE_FINALIZE:
            eng.run(1)
        self._stale()
        return eng.clock(0).a


def analyse(pm: PM3D, a: float, fracs=(0.1, 0.2, 0.3), radii_cells=(1.0, 2.0, 4.0, 8.0)):
    """Axes of the inner Lagrangian sets and enclosed-mass compaction around the densest point
    (pm3d.py:132-159); the reductions over all particles run on the GPU in float64."""
    torch = pm._torch
    lib = _lib.load()
    L, Np = pm.L, pm.Np
    n = Np ** 3
    out = {"a": a}
    dev = f"cuda:{pm.device}"
    A = np.ascontiguousarray(pm.A, dtype=np.float64)
    if getattr(pm, "_core_ids", None) is None:
        keys = torch.empty(n, dtype=torch.int64, device=dev)
        check(lib.pm_rell_keys(Np, L, A.ctypes.data_as(C.c_void_p), keys.data_ptr()), "pm_rell_keys")
        from .engine import sort_u64
        _, perm = sort_u64(keys.cpu().numpy().view(np.uint64), 0, 64)
        pm._core_ids = perm[:30].astype(np.int64)
    pm._flush()
    x, _ = pm._engine.particles(0)
    core = np.sort(pm._core_ids[:27])
    xc = x[torch.as_tensor(core, device=dev)].cpu().numpy()
    rel = (xc - xc[0] + L / 2) % L - L / 2                       # pm3d.py:138-141
    c = (xc[0] + rel.mean(axis=0)) % L
    rm = np.sqrt(6.0)
    set_r = np.array([f * rm for f in fracs], dtype=np.float64)
    radii = np.array([nc * pm.dx for nc in radii_cells], dtype=np.float64)
    nblk = 592
    part = torch.empty((nblk, 34), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    check(lib.pm_analyse_partials(x.data_ptr(), Np, L, A.ctypes.data_as(C.c_void_p),
                                  np.ascontiguousarray(c).ctypes.data_as(C.c_void_p),
                                  set_r.ctypes.data_as(C.c_void_p), radii.ctypes.data_as(C.c_void_p), nblk,
                                  part.data_ptr()), "pm_analyse_partials")
    S = part.cpu().numpy().sum(axis=0)
    fallback = None
    for s, f in enumerate(fracs):
        cnt, s1, s2 = S[10 * s], S[10 * s + 1:10 * s + 4], S[10 * s + 4:10 * s + 10]
        if cnt < 30:                                              # pm3d.py:145
            if fallback is None:
                ids = np.sort(pm._core_ids[:30])
                xf = x[torch.as_tensor(ids, device=dev)].cpu().numpy()
                fallback = (xf - c + L / 2) % L - L / 2
            r = fallback - fallback.mean(axis=0)
            I = r.T @ r / len(r)
            cnt = 30.0
        else:
            mean = s1 / cnt
            M2 = np.array([[s2[0], s2[1], s2[2]], [s2[1], s2[3], s2[4]], [s2[2], s2[4], s2[5]]])
            I = (M2 - cnt * np.outer(mean, mean)) / cnt
        ev = np.sqrt(np.maximum(np.linalg.eigvalsh(I), 0.0)) * np.sqrt(5.0)
        M = pm.m_part * cnt
        axes_phys = a * ev[::-1]
        R_hoop = np.sqrt(0.5 * (axes_phys[0] ** 2 + axes_phys[1] ** 2))
        out[f"axes_{f}"] = axes_phys.tolist()
        out[f"axes_com_{f}"] = ev[::-1].tolist()
        out[f"M_{f}"] = M
        out[f"hoop_{f}"] = 2 * M / max(R_hoop, 1e-30)
    for k, nc in enumerate(radii_cells):
        M = pm.m_part * S[30 + k]
        out[f"m_in_{nc:g}c"] = M
        out[f"C_{nc:g}c"] = 2 * M / (a * nc * pm.dx)
    pm._prime()
    out["rho_max_over_mean"] = float(pm._engine.stats(0).rho_max_over_mean)
    return out
