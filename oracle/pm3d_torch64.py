"""Float64 torch oracle of the pm3d step for large meshes -- TEST INFRASTRUCTURE ONLY.

The numpy oracle (``oracle.pm3d_oracle``) restates ``pbhgr/pbhgr/pm3d.py`` but takes minutes
per step at 512^3.  This module restates the same functions in float64 torch so they run on a
GPU (or on the CPU for small meshes): the CIC deposit as eight ``index_add_`` passes, the
spectral Green's function through ``torch.fft`` (cuFFT in double precision on a GPU), the CIC
interpolation as eight gathers and the KDK leapfrog in a.  It uses no code of ``pbh_b200``.
It is checked against the numpy oracle by ``tests/test_oracle.py`` (CPU, small meshes) and is
the reference for the large-mesh trajectory test in ``tests/test_gpu_large.py``.
Float64 ``index_add_`` on a GPU accumulates with atomics, so its sums are order-dependent at
the 1e-16 level; that is far below every tolerance it is used for.
"""
from __future__ import annotations

import math

import torch

H_I = 5.0                                       # pm3d.py:15
RHO_A3 = 3.0 * H_I ** 2 / (8.0 * math.pi)      # pm3d.py:17


class TorchMesh:
    """Geometry and k-grids of ``PM3D.__init__`` (pm3d.py:27-37) on a torch device."""

    def __init__(self, N: int, L: float, Np: int, smooth: float = 0.0, device="cpu"):
        self.N, self.L, self.Np, self.smooth = int(N), float(L), int(Np), float(smooth)
        self.dx = self.L / self.N
        self.device = torch.device(device)
        f64 = dict(dtype=torch.float64, device=self.device)
        kline = 2.0 * math.pi * torch.fft.fftfreq(self.N, d=self.dx, **f64)
        khalf = 2.0 * math.pi * torch.fft.rfftfreq(self.N, d=self.dx, **f64)
        self.kx = kline.view(-1, 1, 1)
        self.ky = kline.view(1, -1, 1)
        self.kz = khalf.view(1, 1, -1)
        k2 = self.kx ** 2 + self.ky ** 2 + self.kz ** 2
        k2[0, 0, 0] = 1.0
        self.k2 = k2
        self.m_part = RHO_A3 * self.L ** 3 / self.Np ** 3
        self.n_mean = self.Np ** 3 / self.N ** 3

    def _corners(self, X):
        """The 8 (flat node index, weight) pairs of CIC (pm3d.py:76-79, 83-88)."""
        N = self.N
        g = X / self.dx - 0.5
        lo = torch.floor(g)
        f = g - lo
        lo = lo.to(torch.int64)
        i0 = torch.remainder(lo, N)
        i1 = torch.remainder(lo + 1, N)
        for ix, wx in ((i0[:, 0], 1.0 - f[:, 0]), (i1[:, 0], f[:, 0])):
            for iy, wy in ((i0[:, 1], 1.0 - f[:, 1]), (i1[:, 1], f[:, 1])):
                for iz, wz in ((i0[:, 2], 1.0 - f[:, 2]), (i1[:, 2], f[:, 2])):
                    yield (ix * N + iy) * N + iz, wx * wy * wz

    def deposit(self, X):
        """CIC counts per node (pm3d.py:81-89)."""
        rho = torch.zeros(self.N ** 3, dtype=torch.float64, device=self.device)
        for flat, w in self._corners(X):
            rho.index_add_(0, flat, w)
        return rho.view(self.N, self.N, self.N)

    def interp(self, F, X):
        """CIC gather (pm3d.py:91-99)."""
        flat_f = F.reshape(-1)
        out = torch.zeros(X.shape[0], dtype=torch.float64, device=self.device)
        for flat, w in self._corners(X):
            out += flat_f[flat] * w
        return out

    def potential_k(self, delta, a: float):
        """Phi_k = -(3/2) H_i^2 delta_k /(a k^2), optional Gaussian smoothing, zero mode
        removed (pm3d.py:105-109)."""
        phik = (-1.5 * H_I ** 2 / a) * torch.fft.rfftn(delta) / self.k2
        if self.smooth > 0:
            phik = phik * torch.exp(-0.5 * self.k2 * (self.smooth * self.dx) ** 2)
        phik[0, 0, 0] = 0.0
        return phik

    def forces(self, X, a: float):
        """(-grad Phi at the particles, delta) of ``PM3D.forces`` (pm3d.py:101-114); numpy's
        irfftn convention (Hermitian part of the kz = 0, N/2 planes) is what torch's irfftn
        computes as well."""
        N = self.N
        delta = self.deposit(X) / self.n_mean - 1.0
        phik = self.potential_k(delta, a)
        acc = []
        for kc in (self.kx, self.ky, self.kz):
            g = torch.fft.irfftn(-1j * kc * phik, s=(N, N, N))
            acc.append(self.interp(g, X))
            del g
        return torch.stack(acc, dim=-1), delta

    def energies(self, X, P, a: float):
        """(m_p sum p, K, W) at expansion factor a, as ``oracle.pm3d_oracle.energies``: K =
        m_p/(2 a^2) sum p^2 and W = (1/2) rho_b a^3 dx^3 sum_nodes delta Phi, from pm3d's
        equations of motion (pm3d.py:3-6) and its mesh potential (pm3d.py:103-109)."""
        mom = self.m_part * P.sum(dim=0)
        kin = self.m_part / (2.0 * a * a) * float((P * P).sum())
        delta = self.deposit(X) / self.n_mean - 1.0
        phi = torch.fft.irfftn(self.potential_k(delta, a), s=(self.N,) * 3)
        pot = 0.5 * RHO_A3 * self.dx ** 3 * float((delta * phi).sum())
        return mom, kin, pot


def hubble(a: float) -> float:
    return H_I * a ** -1.5                      # pm3d.py:118


class TorchTrajectory:
    """KDK leapfrog in a of ``PM3D.step`` (pm3d.py:117-129)."""

    def __init__(self, mesh: TorchMesh, x, p):
        self.mesh = mesh
        self.x = torch.as_tensor(x, dtype=torch.float64).to(mesh.device).clone()
        self.p = torch.as_tensor(p, dtype=torch.float64).to(mesh.device).clone()
        self.acc = None
        self.acc_a = None

    def step(self, a: float, da: float):
        m = self.mesh
        if self.acc is None or self.acc_a != a:                     # pm3d.py:119-120
            self.acc, _ = m.forces(self.x, a)
        self.p += (0.5 * da / (a * hubble(a))) * self.acc            # pm3d.py:122
        a_mid = a + 0.5 * da                                         # pm3d.py:123-124
        self.x = torch.remainder(self.x + (da / (a_mid ** 3 * hubble(a_mid))) * self.p, m.L)
        a_new = a + da                                               # pm3d.py:125-127
        acc, delta = m.forces(self.x, a_new)
        self.p += (0.5 * da / (a_new * hubble(a_new))) * acc
        self.acc, self.acc_a = acc, a_new                            # pm3d.py:128
        return a_new, delta
