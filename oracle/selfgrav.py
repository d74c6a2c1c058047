"""Oracle for the self-gravity path (TEST INFRASTRUCTURE ONLY).

* accel / potential: the C restatement in allpairs.c (sequential j order),
  following `beschleunigung` (reference backend/selfgrav_kernel.py:222-260).
* kdk: the leapfrog of `selfgrav_kernel` (selfgrav_kernel.py:333-419) and of
  `referenz` (test_selfgrav.py:66-88): kick(0.5 dt), drift(dt), force,
  kick(0.5 dt) per step.
* yoshida4: the same KDK substep composed with Yoshida weights w1, w0, w1
  (nbody_kernel.py:64-65).
* energy: Plummer energy with the self terms removed (test_selfgrav.py:54-63).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        dp = ctypes.c_void_p
        for name in ("oracle_allpairs_accel", "oracle_allpairs_absterm", "oracle_allpairs_potential"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_int, dp, ctypes.c_int64, dp, ctypes.c_int64, dp, ctypes.c_double,
                          ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def threads_default() -> int:
    return int(os.environ.get("SSS_ORACLE_THREADS", os.cpu_count() or 1))


def _rec(a):
    a = np.ascontiguousarray(a, np.float64)
    if a.ndim != 2 or a.shape[1] != 4:
        raise ValueError("records must be (n, 4) float64")
    return a


def accel(src4, tgt4, eps2, dim=3, threads=None):
    """(n_tgt, 4) accelerations, sequential source order per target."""
    s, t = _rec(src4), _rec(tgt4)
    out = np.zeros_like(t)
    lib().oracle_allpairs_accel(dim, s.ctypes.data, len(s), t.ctypes.data, len(t), out.ctypes.data,
                                float(eps2), threads or threads_default())
    return out


def absterm(src4, tgt4, eps2, dim=3, threads=None):
    """sum_j |term_j| per component: the scale of summation rounding."""
    s, t = _rec(src4), _rec(tgt4)
    out = np.zeros_like(t)
    lib().oracle_allpairs_absterm(dim, s.ctypes.data, len(s), t.ctypes.data, len(t), out.ctypes.data,
                                  float(eps2), threads or threads_default())
    return out


def potential(src4, tgt4, eps2, dim=3, threads=None):
    s, t = _rec(src4), _rec(tgt4)
    out = np.zeros(len(t))
    lib().oracle_allpairs_potential(dim, s.ctypes.data, len(s), t.ctypes.data, len(t),
                                    out.ctypes.data, float(eps2), threads or threads_default())
    return out


def records(x, y, z=None, gm=None):
    n = len(x)
    r = np.zeros((n, 4))
    r[:, 0] = x
    r[:, 1] = y
    if z is not None:
        r[:, 2] = z
    if gm is not None:
        r[:, 3] = gm
    return r


YOSHIDA_W1 = 1.0 / (2.0 - 2.0 ** (1.0 / 3.0))          # nbody_kernel.py:64
YOSHIDA_W0 = -(2.0 ** (1.0 / 3.0)) / (2.0 - 2.0 ** (1.0 / 3.0))  # :65


def integrate(pos, vel, gm, eps2, dt, steps, dim=3, n_src=None, weights=(1.0,), threads=None,
              snapshots=False):
    """KDK substeps (selfgrav_kernel.py:333-419) composed with `weights`.

    pos, vel: (n_all, 3) f64; bodies [0, n_src) are sources, the rest
    massless tracers. Returns (pos, vel, acc[, snaps]) with snaps the f32
    rows of selfgrav_kernel's snapshot layout after every step."""
    pos = np.array(pos, np.float64, copy=True)
    vel = np.array(vel, np.float64, copy=True)
    n_all = len(pos)
    n_src = n_all if n_src is None else n_src
    rec = np.zeros((n_all, 4))

    def force():
        rec[:, :3] = pos
        rec[:n_src, 3] = gm
        rec[n_src:, 3] = 0.0
        return accel(rec[:n_src], rec, eps2, dim=dim, threads=threads)[:, :3]

    acc = force()
    snaps = []
    for _ in range(steps):
        for w in weights:
            h = w * dt
            vel += acc * (0.5 * h)
            pos += vel * h
            acc = force()
            vel += acc * (0.5 * h)
        if snapshots:
            d = dim
            row = [pos[:n_src, k] for k in range(d)] + [vel[:n_src, k] for k in range(d)] + \
                  [pos[n_src:, k] for k in range(d)]
            snaps.append(np.concatenate(row).astype(np.float32))
    out = (pos, vel, acc)
    if snapshots:
        out = out + (np.array(snaps),)
    return out


def energy(pos, vel, mass, G, eps2, dim=3, threads=None):
    """Kinetic + Plummer potential energy, self terms removed
    (test_selfgrav.py:54-63)."""
    kin = 0.5 * float((mass * (vel[:, :dim] ** 2).sum(1)).sum())
    rec = records(pos[:, 0], pos[:, 1], pos[:, 2] if dim == 3 else None, G * mass)
    phi = potential(rec, rec, eps2, dim=dim, threads=threads)
    pot = 0.5 * float((mass * phi).sum()) + 0.5 * G * float((mass * mass).sum()) / np.sqrt(eps2)
    return kin + pot
