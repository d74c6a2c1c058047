"""Oracle for the batched small systems (TEST INFRASTRUCTURE ONLY).

Per system: the all-pairs force a_i = sum_{j != i} G m_j d / (|d|^2 +
eps2)^1.5 (the reference's pair formula, selfgrav_kernel.py:247-255) and
fixed-step Yoshida-4 as three KDK substeps (nbody_kernel.py:64-65), in f64
NumPy, plus the system's energy."""
from __future__ import annotations

import numpy as np

W1 = 1.0 / (2.0 - 2.0 ** (1.0 / 3.0))
W0 = -(2.0 ** (1.0 / 3.0)) / (2.0 - 2.0 ** (1.0 / 3.0))


def accel(pos, mass, G, eps2=0.0):
    d = pos[:, None, :] - pos[:, :, None]          # d[c, i, j] = x_j - x_i
    r2 = (d * d).sum(0) + eps2
    np.fill_diagonal(r2, 1.0)
    inv3 = r2 ** -1.5
    np.fill_diagonal(inv3, 0.0)
    return (G * mass[None, None, :] * inv3[None] * d).sum(2)


def yoshida(pos, vel, mass, G, dt, steps, eps2=0.0):
    pos, vel = pos.astype(np.float64).copy(), vel.astype(np.float64).copy()
    a = accel(pos, mass, G, eps2)
    for _ in range(steps):
        for w in (W1, W0, W1):
            h = w * dt
            vel += a * (0.5 * h)
            pos += vel * h
            a = accel(pos, mass, G, eps2)
            vel += a * (0.5 * h)
    return pos, vel


def energy(pos, vel, mass, G, eps2=0.0):
    kin = 0.5 * np.sum(mass * (vel * vel).sum(0))
    d = pos[:, None, :] - pos[:, :, None]
    r = np.sqrt((d * d).sum(0) + eps2)
    iu = np.triu_indices(len(mass), 1)
    return kin - G * np.sum(mass[iu[0]] * mass[iu[1]] / r[iu])
