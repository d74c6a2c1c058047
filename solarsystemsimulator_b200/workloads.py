"""Seeded synthetic workloads of the benchmark configurations.

No dataset is involved: every configuration is generated from a seed with
the shapes, sizes and value distributions the configuration states.
"""
from __future__ import annotations

import numpy as np

SEED_STRUCTURE = 20260303   # self-gravitating structure formation


def zeldovich_displacement(ngrid: int, sigma_delta: float, index: float, seed: int):
    """Zel'dovich displacement field psi on an ngrid^3 periodic unit lattice.

    delta_k is a Gaussian random field with P(k) ~ k^index (white noise
    shaped in Fourier space), normalised to rms density contrast
    sigma_delta; psi_k = i k delta_k / k^2 so that delta = -div(psi).
    Returns psi with shape (3, ngrid, ngrid, ngrid)."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((ngrid, ngrid, ngrid))
    wk = np.fft.rfftn(white)
    k1 = 2 * np.pi * np.fft.fftfreq(ngrid, d=1.0 / ngrid)
    kr = 2 * np.pi * np.fft.rfftfreq(ngrid, d=1.0 / ngrid)
    kx, ky, kz = np.meshgrid(k1, k1, kr, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = k2 ** (index / 4.0)          # sqrt(P) = k^(index/2) = (k^2)^(index/4)
    amp[0, 0, 0] = 0.0
    dk = wk * amp
    delta = np.fft.irfftn(dk, s=(ngrid,) * 3)
    dk *= sigma_delta / delta.std()
    psi = np.empty((3, ngrid, ngrid, ngrid))
    for c, kc in enumerate((kx, ky, kz)):
        psi[c] = np.fft.irfftn(1j * kc * dk / k2, s=(ngrid,) * 3)
    return psi


def _interp_periodic(field: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Trilinear interpolation of a cell-centred periodic field at q in [0,1)^3."""
    n = field.shape[-1]
    g = q * n - 0.5
    i0 = np.floor(g).astype(np.int64)
    t = g - i0
    out = np.zeros((field.shape[0], len(q)))
    for dx in (0, 1):
        wx = t[:, 0] if dx else 1 - t[:, 0]
        ix = (i0[:, 0] + dx) % n
        for dy in (0, 1):
            wy = t[:, 1] if dy else 1 - t[:, 1]
            iy = (i0[:, 1] + dy) % n
            for dz in (0, 1):
                wz = t[:, 2] if dz else 1 - t[:, 2]
                iz = (i0[:, 2] + dz) % n
                out += field[:, ix, iy, iz] * (wx * wy * wz)
    return out


def structure_formation(n_side: int = 64, n_tracer: int = 524_288, sigma_delta: float = 0.01,
                        index: float = -2.0, seed: int = SEED_STRUCTURE):
    """Self-gravitating structure formation: n_side^3 equal-mass sources in
    the unit cube on a lattice displaced by Zel'dovich displacements from
    P(k) ~ k^index with rms density contrast sigma_delta, cold start (zero
    velocities), plus n_tracer massless tracers drawn uniformly and displaced
    by the same field. Total mass 1.

    Returns dict with pos (n,3), mass (n,), tracer_pos (T,3)."""
    psi = zeldovich_displacement(n_side, sigma_delta, index, seed)
    i = (np.arange(n_side) + 0.5) / n_side
    qx, qy, qz = np.meshgrid(i, i, i, indexing="ij")
    q = np.stack([qx.ravel(), qy.ravel(), qz.ravel()], 1)
    pos = q + np.stack([psi[c].ravel() for c in range(3)], 1)
    rng = np.random.default_rng(seed + 1)
    qt = rng.uniform(0.0, 1.0, (n_tracer, 3))
    tpos = qt + _interp_periodic(psi, qt).T
    n = len(pos)
    return {"pos": pos, "mass": np.full(n, 1.0 / n), "tracer_pos": tpos}
