"""Oracle for the 2-D isolated particle mesh (TEST INFRASTRUCTURE ONLY).

NumPy restatement of the reference's backend/pm_kernel.py: force-kernel
transforms (:34-60), CIC deposit (:63-90) and gather (:93-107), grid
geometry (:110-124), field (:127-147), and the KDK loop of NBodyPM
(:212-280) with its kernel cache rule. f64 with NumPy's FFT.
"""
from __future__ import annotations

import numpy as np

G_AU = 4 * np.pi * np.pi


def build_force_kernels(grid_n, h, eps2, G=G_AU):
    n_pad = 2 * grid_n
    off = np.arange(n_pad, dtype=np.float64)
    off = np.where(off < grid_n, off, off - n_pad)
    dx = (off * h)[:, None]
    dy = (off * h)[None, :]
    r2 = dx * dx + dy * dy + eps2
    inv_r3 = 1.0 / (r2 * np.sqrt(r2))
    return np.fft.rfft2((-G) * dx * inv_r3), np.fft.rfft2((-G) * dy * inv_r3)


def _corners(gx, gy, grid_n, x0, y0, h):
    fx = (gx - x0) / h
    fy = (gy - y0) / h
    i = np.clip(np.floor(fx).astype(np.int32), 0, grid_n - 2)
    j = np.clip(np.floor(fy).astype(np.int32), 0, grid_n - 2)
    return i, j, fx - i, fy - j


def cic_deposit(gx, gy, gm, grid_n, x0, y0, h):
    i, j, tx, ty = _corners(gx, gy, grid_n, x0, y0, h)
    idx = np.concatenate([i * grid_n + j, (i + 1) * grid_n + j, i * grid_n + (j + 1), (i + 1) * grid_n + (j + 1)])
    w = np.concatenate([gm * (1 - tx) * (1 - ty), gm * tx * (1 - ty), gm * (1 - tx) * ty, gm * tx * ty])
    return np.bincount(idx, weights=w, minlength=grid_n * grid_n).reshape(grid_n, grid_n)


def cic_gather(feld, gx, gy, grid_n, x0, y0, h):
    i, j, tx, ty = _corners(gx, gy, grid_n, x0, y0, h)
    f = feld.ravel()
    return (f[i * grid_n + j] * (1 - tx) * (1 - ty) + f[(i + 1) * grid_n + j] * tx * (1 - ty)
            + f[i * grid_n + (j + 1)] * (1 - tx) * ty + f[(i + 1) * grid_n + (j + 1)] * tx * ty)


def grid_fuer(gx, gy, grid_n, rand_zellen=3.0):
    spanne = max(float(gx.max()) - float(gx.min()), float(gy.max()) - float(gy.min()), 1e-30)
    h = spanne / (grid_n - 2 * rand_zellen)
    return float(gx.min()) - rand_zellen * h, float(gy.min()) - rand_zellen * h, h


def pm_force_field(gx, gy, gm, grid_n, x0, y0, h, eps2, G=G_AU, kernels=None):
    if kernels is None:
        kernels = build_force_kernels(grid_n, h, eps2, G)
    fkx, fky = kernels
    n_pad = 2 * grid_n
    rho_pad = np.zeros((n_pad, n_pad))
    rho_pad[:grid_n, :grid_n] = cic_deposit(gx, gy, gm, grid_n, x0, y0, h)
    fr = np.fft.rfft2(rho_pad)
    ax = np.fft.irfft2(fr * fkx, s=(n_pad, n_pad))[:grid_n, :grid_n]
    ay = np.fft.irfft2(fr * fky, s=(n_pad, n_pad))[:grid_n, :grid_n]
    return ax, ay


def pm_accelerations(gx, gy, gm, grid_n, x0, y0, h, eps2, G=G_AU):
    ax, ay = pm_force_field(gx, gy, gm, grid_n, x0, y0, h, eps2, G)
    return cic_gather(ax, gx, gy, grid_n, x0, y0, h), cic_gather(ay, gx, gy, grid_n, x0, y0, h)


def kdk(x, y, vx, vy, m, tracer, dt, steps, grid_n, soft_cells=1.5, rand_cells=4.0, soft_floor=0.0, G=G_AU):
    """NBodyPM.load_state + step_batch (pm_kernel.py:212-280)."""
    x, y, vx, vy = (np.array(a, np.float64, copy=True) for a in (x, y, vx, vy))
    tx, ty, tvx, tvy = (np.array(a, np.float64, copy=True) for a in tracer)
    cache = {"h": None, "k": None}

    def accel():
        x0, y0, h = grid_fuer(x, y, grid_n, rand_cells)
        eps = max(soft_cells * h, soft_floor)
        if cache["h"] is None or abs(h - cache["h"]) > 1e-6 * h:
            cache["k"] = build_force_kernels(grid_n, h, eps * eps, G)
            cache["h"] = h
        fx, fy = pm_force_field(x, y, m, grid_n, x0, y0, h, eps * eps, G, cache["k"])
        return (cic_gather(fx, x, y, grid_n, x0, y0, h), cic_gather(fy, x, y, grid_n, x0, y0, h),
                cic_gather(fx, tx, ty, grid_n, x0, y0, h), cic_gather(fy, tx, ty, grid_n, x0, y0, h))

    ax, ay, tax, tay = accel()
    hdt = 0.5 * dt
    rows = []
    for _ in range(steps):
        vx += hdt * ax; vy += hdt * ay
        x += dt * vx; y += dt * vy
        tvx += hdt * tax; tvy += hdt * tay
        tx += dt * tvx; ty += dt * tvy
        ax, ay, tax, tay = accel()
        vx += hdt * ax; vy += hdt * ay
        tvx += hdt * tax; tvy += hdt * tay
        rows.append(np.concatenate([x, y, vx, vy, tx, ty]).astype(np.float32))
    return np.array(rows), np.concatenate([x, y, vx, vy])
