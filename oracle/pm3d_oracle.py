"""CPU oracle for the pm3d particle-mesh path -- TEST INFRASTRUCTURE ONLY.

This module is a float64 numpy restatement of the reference algorithm in
``pbhgr/pbhgr/pm3d.py`` (uniquehuman/pbh).  It is imported only by ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``; the
product package ``pbh_b200`` never imports it.  Every function names the
reference lines it restates.  It is pinned against the reference itself by the
golden fixtures in ``tests/golden/`` (generated by ``tests/golden/make_golden.py``
importing the unmodified reference) and checked by ``tests/test_oracle.py``.

Units (``pm3d.py:3-9``): G = c = 1, a_i = 1, H_i = 5, comoving box [0, L)^3,
canonical momentum p = a^2 dx/dt.
"""
from __future__ import annotations

import numpy as np

# pm3d.py:15-17
H_I = 5.0
T_I = 2.0 / (3.0 * H_I)
RHO_A3 = 3.0 * H_I ** 2 / (8.0 * np.pi)


def zeldovich_axes(e: float, p: float) -> np.ndarray:
    """Axis lengths A_i ~ lambda_i^(-1/2) normalised to prod A = 1 (pm3d.py:20-23)."""
    lam = np.array([1.0 + 3.0 * e + p, 1.0 - 2.0 * p, 1.0 - 3.0 * e + p]) / 3.0
    ax = 1.0 / np.sqrt(lam)
    return ax / np.cbrt(np.prod(ax))


class Mesh:
    """Mesh geometry and k-grids of ``PM3D.__init__`` (pm3d.py:27-37)."""

    def __init__(self, N: int, L: float, Np: int, smooth: float = 0.0):
        self.N, self.L, self.Np, self.smooth = int(N), float(L), int(Np), float(smooth)
        self.dx = self.L / self.N
        kline = 2.0 * np.pi * np.fft.fftfreq(self.N, d=self.dx)
        khalf = 2.0 * np.pi * np.fft.rfftfreq(self.N, d=self.dx)
        self.kx = kline[:, None, None] * np.ones((1, self.N, khalf.size))
        self.ky = kline[None, :, None] * np.ones((self.N, 1, khalf.size))
        self.kz = khalf[None, None, :] * np.ones((self.N, self.N, 1))
        self.k2 = self.kx ** 2 + self.ky ** 2 + self.kz ** 2
        self.k2[0, 0, 0] = 1.0
        self.m_part = RHO_A3 * self.L ** 3 / self.Np ** 3

    @property
    def n_mean(self) -> float:
        return self.Np ** 3 / self.N ** 3


def cic_split(X1: np.ndarray, dx: float, N: int):
    """Lower node, upper node and fraction along one axis (pm3d.py:76-79).

    Node i sits at (i + 1/2) dx, so g = X/dx - 1/2 measures position in node
    units; the particle lies between nodes floor(g) and floor(g) + 1.
    """
    g = X1 / dx - 0.5
    lo = np.floor(g).astype(np.int64)
    return lo % N, (lo + 1) % N, g - lo


def _corners(X: np.ndarray, dx: float, N: int):
    """The 8 (flat node index, weight) pairs of CIC (pm3d.py:83-88, 93-98)."""
    sx = cic_split(X[:, 0], dx, N)
    sy = cic_split(X[:, 1], dx, N)
    sz = cic_split(X[:, 2], dx, N)
    for ix, wx in ((sx[0], 1.0 - sx[2]), (sx[1], sx[2])):
        for iy, wy in ((sy[0], 1.0 - sy[2]), (sy[1], sy[2])):
            for iz, wz in ((sz[0], 1.0 - sz[2]), (sz[1], sz[2])):
                yield (ix * N + iy) * N + iz, wx * wy * wz


def deposit(X: np.ndarray, N: int, dx: float) -> np.ndarray:
    """Particle counts per mesh node, CIC assignment (pm3d.py:81-89)."""
    rho = np.zeros(N ** 3)
    for flat, w in _corners(X, dx, N):
        rho += np.bincount(flat, weights=w, minlength=N ** 3)
    return rho.reshape(N, N, N)


def interp(F: np.ndarray, X: np.ndarray, N: int, dx: float) -> np.ndarray:
    """CIC gather of a mesh field at the particles (pm3d.py:91-99)."""
    flatF = F.reshape(-1)
    out = np.zeros(len(X))
    for flat, w in _corners(X, dx, N):
        out += flatF[flat] * w
    return out


def _irfftn(spec: np.ndarray, N: int) -> np.ndarray:
    # numpy's multi-axis C2R: complex inverse over axes 0,1 then C2R over axis 2.
    return np.fft.irfftn(spec, s=(N, N, N), axes=(0, 1, 2))


def potential_k(mesh: Mesh, dk: np.ndarray, a: float) -> np.ndarray:
    """Phi_k = -(3/2) H_i^2 delta_k /(a k^2), optional Gaussian smoothing,
    zero mode removed (pm3d.py:106-109)."""
    phik = (-1.5 * H_I ** 2 / a) * dk / mesh.k2
    if mesh.smooth > 0:
        phik = phik * np.exp(-0.5 * mesh.k2 * (mesh.smooth * mesh.dx) ** 2)
    phik[0, 0, 0] = 0.0
    return phik


def force_grids(mesh: Mesh, delta: np.ndarray, a: float):
    """The three mesh fields -dPhi/dx_i (pm3d.py:105-112)."""
    dk = np.fft.rfftn(delta)
    phik = potential_k(mesh, dk, a)
    return [_irfftn(-1j * kc * phik, mesh.N) for kc in (mesh.kx, mesh.ky, mesh.kz)]


def force_grids_fd(mesh: Mesh, delta: np.ndarray, a: float, order: int):
    """-dPhi/dx_i by central differences of the potential in real space, the finite-difference
    alternative to the spectral gradient of pm3d.py:110-112 (which has no such option): order 2,
    -(Phi(x+dx) - Phi(x-dx))/(2dx); order 4, -(8[Phi(x+dx) - Phi(x-dx)] - [Phi(x+2dx) -
    Phi(x-2dx)])/(12dx).  Phi is the reference's potential (pm3d.py:105-109)."""
    phi = _irfftn(potential_k(mesh, np.fft.rfftn(delta), a), mesh.N)
    out = []
    for ax in range(3):
        d1 = np.roll(phi, -1, axis=ax) - np.roll(phi, 1, axis=ax)
        if order == 2:
            out.append(-d1 / (2.0 * mesh.dx))
        else:
            d2 = np.roll(phi, -2, axis=ax) - np.roll(phi, 2, axis=ax)
            out.append(-(8.0 * d1 - d2) / (12.0 * mesh.dx))
    return out


def density_contrast(mesh: Mesh, X: np.ndarray) -> np.ndarray:
    """delta = n/n_mean - 1 from the CIC counts (pm3d.py:103-104)."""
    return deposit(X, mesh.N, mesh.dx) / mesh.n_mean - 1.0


def accelerations(mesh: Mesh, X: np.ndarray, a: float):
    """``PM3D.forces``: (-grad Phi at the particles, delta) (pm3d.py:101-114)."""
    delta = density_contrast(mesh, X)
    grids = force_grids(mesh, delta, a)
    acc = np.stack([interp(g, X, mesh.N, mesh.dx) for g in grids], axis=-1)
    return acc, delta


def hubble(a: float) -> float:
    """EdS: H = H_i a^(-3/2) (pm3d.py:5, 118)."""
    return H_I * a ** -1.5


def energies(mesh: Mesh, x: np.ndarray, p: np.ndarray, a: float):
    """Total momentum, kinetic and mesh potential energy at expansion factor ``a``.

    ``pm3d.py`` has no energy diagnostic; this follows from its equations of motion
    (pm3d.py:3-6: p = a^2 dx/dt, dp/dt = -grad Phi, lap Phi = (3/2) H_i^2 delta / a) and its
    mesh potential (pm3d.py:103-109): K = m_p/(2 a^2) sum p^2 (peculiar velocity p/a) and
    W = (1/2) rho_b a^3 dx^3 sum_nodes delta Phi.  They obey the Layzer-Irvine equation
    d[a (K + W)]/da = -K.
    """
    mom = mesh.m_part * p.sum(axis=0)
    kin = mesh.m_part / (2.0 * a * a) * float((p * p).sum())
    delta = density_contrast(mesh, x)
    phi = _irfftn(potential_k(mesh, np.fft.rfftn(delta), a), mesh.N)
    pot = 0.5 * RHO_A3 * mesh.dx ** 3 * float((delta * phi).sum())
    return mom, kin, pot


def layzer_irvine(samples):
    """a (K + W) + int K da - a0 (K0 + W0) at the last of ``samples`` [(a, K, W), ...], the
    integral by the trapezoid rule between consecutive samples."""
    a0, k0, w0 = samples[0]
    integral = 0.0
    for (a1, k1, _), (a2, k2, _) in zip(samples[:-1], samples[1:]):
        integral += 0.5 * (k1 + k2) * (a2 - a1)
    a, k, w = samples[-1]
    return a * (k + w) + integral - a0 * (k0 + w0)


class Trajectory:
    """Particle state and the KDK leapfrog in a of ``PM3D.step`` (pm3d.py:117-129)."""

    def __init__(self, mesh: Mesh, x: np.ndarray, p: np.ndarray):
        self.mesh = mesh
        self.x = np.array(x, dtype=np.float64)
        self.p = np.array(p, dtype=np.float64)
        self.acc = None
        self.acc_a = None

    def step(self, a: float, da: float):
        m = self.mesh
        if self.acc is None or self.acc_a != a:          # pm3d.py:119-120
            self.acc, _ = accelerations(m, self.x, a)
        self.p = self.p + (0.5 * da / (a * hubble(a))) * self.acc          # pm3d.py:122
        a_mid = a + 0.5 * da                                                # pm3d.py:123-124
        self.x = (self.x + da * self.p / (a_mid ** 3 * hubble(a_mid))) % m.L
        a_new = a + da                                                      # pm3d.py:125-127
        acc, delta = accelerations(m, self.x, a_new)
        self.p = self.p + (0.5 * da / (a_new * hubble(a_new))) * acc
        self.acc, self.acc_a = acc, a_new                                   # pm3d.py:128
        return a_new, delta


# --------------------------------------------------------------------- initial data
def lattice(Np: int, L: float) -> np.ndarray:
    """Quiet-start lattice, centred coordinates, 'ij' order (pm3d.py:64-65)."""
    q1 = (np.arange(Np) + 0.5) * (L / Np) - L / 2
    g = np.meshgrid(q1, q1, q1, indexing="ij")
    return np.stack(g, axis=-1).reshape(-1, 3)


def cell_centres(N: int, L: float):
    """Centred cell coordinates of the mesh (pm3d.py:42-43)."""
    xg = (np.arange(N) + 0.5) * (L / N) - L / 2
    return np.meshgrid(xg, xg, xg, indexing="ij")


def zeldovich_from_delta_k(mesh: Mesh, dk: np.ndarray, A: np.ndarray):
    """Displacement field, lattice and particles from a linear density
    spectrum at a = 1 (pm3d.py:59-72, starting after delta_k is formed).

    Returns dict(x, p, q, delta_lin, r_ell_q, A)."""
    N, L = mesh.N, mesh.L
    dk = dk.copy()
    dk[0, 0, 0] = 0.0                                         # pm3d.py:60
    phik = -dk / mesh.k2                                      # pm3d.py:61
    psi = [-_irfftn(1j * kc * phik, N) for kc in (mesh.kx, mesh.ky, mesh.kz)]   # pm3d.py:62
    Q = lattice(mesh.Np, L)
    at = (Q + L / 2) % L
    disp = np.stack([interp(f, at, N, mesh.dx) for f in psi], axis=-1)         # pm3d.py:66
    return dict(x=(Q + disp + L / 2) % L, p=H_I * disp, q=Q,                   # pm3d.py:67-69
                delta_lin=_irfftn(dk, N),                                      # pm3d.py:70
                r_ell_q=np.sqrt(np.sum((Q / A) ** 2, axis=1)), A=np.asarray(A))  # pm3d.py:71-72


def zeta_ic(mesh: Mesh, rng, mu, profile_spline, e=0.0, p=0.0, tail_rms=0.0, tail_k=(2.0, 10.0)):
    """``PM3D.make_ic`` (pm3d.py:40-73): curvature profile on the ellipsoidal
    radius, optional flat-in-ln-k tail drawn from ``rng``, delta_k = 0.4 k^2 zeta_k/H_i^2."""
    N, L = mesh.N, mesh.L
    X, Y, Z = cell_centres(N, L)
    A = zeldovich_axes(e, p)
    r_ell = np.sqrt((X / A[0]) ** 2 + (Y / A[1]) ** 2 + (Z / A[2]) ** 2)          # pm3d.py:45
    zk = np.fft.rfftn(mu * profile_spline(np.minimum(r_ell, profile_spline.x[-1])))  # pm3d.py:46-47
    tail_grid = 0.0
    if tail_rms > 0:                                                             # pm3d.py:48-56
        kk = np.sqrt(mesh.k2)
        kk[0, 0, 0] = 0.0
        band = (kk >= tail_k[0]) & (kk <= tail_k[1])
        Pk = np.zeros_like(kk)
        Pk[band] = 2 * np.pi ** 2 * tail_rms ** 2 / (np.maximum(kk[band], 1e-30) ** 3 * np.log(tail_k[1] / tail_k[0]))
        tk = np.fft.rfftn(rng.standard_normal((N, N, N))) * np.sqrt(Pk * N ** 3 / L ** 3)
        tail_grid = float(np.std(_irfftn(tk, N)))
        zk = zk + tk
    dk = 0.4 * mesh.k2 / H_I ** 2 * zk                                           # pm3d.py:59
    out = zeldovich_from_delta_k(mesh, dk, A)
    out["tail_rms_grid"] = tail_grid
    return out


# --------------------------------------------------------------------- diagnostics
def _periodic_mean(xs: np.ndarray, L: float) -> np.ndarray:
    """Mean position unwrapped about the first member (pm3d.py:138-140)."""
    rel = (xs - xs[0] + L / 2) % L - L / 2
    return (xs[0] + rel.mean(axis=0)) % L


def analyse(mesh: Mesh, x: np.ndarray, r_ell_q: np.ndarray, a: float,
            fracs=(0.1, 0.2, 0.3), radii_cells=(1.0, 2.0, 4.0, 8.0), order=None):
    """Peak diagnostics of ``analyse`` (pm3d.py:132-159).

    ``order`` is the argsort of r_ell_q used to pick the 27 (and fallback 30)
    innermost Lagrangian particles; by default a stable argsort (ties broken by
    lattice index)."""
    L = mesh.L
    out = {"a": a}
    if order is None:
        order = np.argsort(r_ell_q, kind="stable")
    rm = np.sqrt(6.0)
    core = np.zeros(len(x), bool)
    core[order[:27]] = True
    c = _periodic_mean(x[core], L)
    rel_all = (x - c + L / 2) % L - L / 2
    for f in fracs:
        sel = r_ell_q < f * rm
        if sel.sum() < 30:
            sel = np.zeros(len(x), bool)
            sel[order[:30]] = True
        rel = rel_all[sel]
        rel = rel - rel.mean(axis=0)
        I = rel.T @ rel / len(rel)
        ev = np.sqrt(np.maximum(np.linalg.eigvalsh(I), 0.0)) * np.sqrt(5.0)
        M = mesh.m_part * sel.sum()
        axes_phys = a * ev[::-1]
        R_hoop = np.sqrt(0.5 * (axes_phys[0] ** 2 + axes_phys[1] ** 2))
        out[f"axes_{f}"] = axes_phys.tolist()
        out[f"axes_com_{f}"] = ev[::-1].tolist()
        out[f"M_{f}"] = M
        out[f"hoop_{f}"] = 2 * M / max(R_hoop, 1e-30)
    r_com = np.sqrt(np.sum(rel_all ** 2, axis=1))
    for nc in radii_cells:
        M = mesh.m_part * np.count_nonzero(r_com < nc * mesh.dx)
        out[f"m_in_{nc:g}c"] = M
        out[f"C_{nc:g}c"] = 2 * M / (a * nc * mesh.dx)
    out["rho_max_over_mean"] = float(np.max(deposit(x, mesh.N, mesh.dx)) / mesh.n_mean)
    return out
