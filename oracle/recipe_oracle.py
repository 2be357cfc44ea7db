"""CPU oracle for the benchmark peak recipe -- TEST INFRASTRUCTURE ONLY.

The benchmark configurations describe a peak as a Gaussian linear density
field delta(x) = delta0 exp(-sum x_i^2 / 2 R_i^2) plus seeded Gaussian noise
with P(k) ~ k^-2 scaled to a fixed fraction of delta0.  ``PM3D.make_ic``
(``pbhgr/pbhgr/pm3d.py:40-73``) cannot express that field (it takes a
curvature profile), so this module builds delta_k in float64 numpy and then
follows the reference's own Zel'dovich tail (``pm3d.py:59-72``, restated in
``oracle.pm3d_oracle.zeldovich_from_delta_k``).  The noise draw follows the
reference's pattern ``rng.standard_normal((N, N, N))`` -> ``rfftn`` -> times
sqrt(P) (``pm3d.py:53-54``), drawing from the run's own generator
``default_rng(seed)`` (``pm3d.py:36``).

The delta_k construction has no counterpart in the reference, so it has no
golden vectors of its own; the Zel'dovich tail it feeds is pinned by the
``zeta_*`` fixtures.
"""
from __future__ import annotations

import numpy as np

from .pm3d_oracle import Mesh, cell_centres, zeldovich_from_delta_k


def gaussian_peak_delta_k(mesh: Mesh, R, delta0: float, noise_frac: float, rng) -> np.ndarray:
    """Spectrum of delta0 exp(-sum x_i^2/2R_i^2) + noise on the cell-centred grid."""
    N, L = mesh.N, mesh.L
    X, Y, Z = cell_centres(N, L)
    R = np.asarray(R, dtype=np.float64)
    field = delta0 * np.exp(-(X ** 2 / (2 * R[0] ** 2) + Y ** 2 / (2 * R[1] ** 2) + Z ** 2 / (2 * R[2] ** 2)))
    dk = np.fft.rfftn(field)
    if noise_frac > 0:
        nk = np.fft.rfftn(rng.standard_normal((N, N, N)))
        shape = 1.0 / np.sqrt(mesh.k2)          # sqrt(P), P = k^-2
        shape[0, 0, 0] = 0.0
        nk = nk * shape
        rms = float(np.std(np.fft.irfftn(nk, s=(N, N, N), axes=(0, 1, 2))))
        dk = dk + nk * (noise_frac * delta0 / rms)
    return dk


def recipe_ic(mesh: Mesh, R, delta0: float, noise_frac: float, seed: int):
    """Particles of the recipe peak: dict(x, p, q, delta_lin, r_ell_q, A)."""
    rng = np.random.default_rng(seed)
    dk = gaussian_peak_delta_k(mesh, R, delta0, noise_frac, rng)
    R = np.asarray(R, dtype=np.float64)
    A = R / np.cbrt(np.prod(R))
    return zeldovich_from_delta_k(mesh, dk, A)
