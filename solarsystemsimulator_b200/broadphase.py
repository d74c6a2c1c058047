"""Asteroid x asteroid collision broadphase on one B200.

Drop-in for the detection layer of the reference's backend/film_producer.py
(`Erkennungskarte`, `_zellschluessel`, `bounce_suche`, `NACHBARN`, `CHUNK`).
The pair search runs in libsss (`sss_broadphase`); the
hit list is bit-exact against the reference's `_hits` on the same f32
snapshot (same pairs, same (i, j) orientation, same order).

    karte = Erkennungskarte(dev, is_ast, -np.inf, np.inf)
    karte.stammdaten(vis, real_r)
    hits, kand = karte.bounce_hits(gx, gy, gvx, gvy, dt_y, h, halo)

`gx..gvy` may be NumPy arrays or CUDA tensors (f32).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

NACHBARN = ((0, 0), (1, 0), (0, 1), (1, 1), (1, -1))   # film_producer.py:155
CHUNK = 4_000_000                                     # film_producer.py:163 (no chunking needed here)


def _dev_f32(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float32).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(device)


def _dev_u8(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return (a != 0).to(device=device, dtype=torch.uint8).contiguous()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a) != 0, dtype=np.uint8)).to(device)


def _dev_flags(a, device) -> torch.Tensor:
    """Per-call flag bytes: a contiguous uint8 tensor on the device is passed
    as it is (the kernels test a byte for nonzero), anything else as _dev_u8."""
    if isinstance(a, torch.Tensor) and a.dtype == torch.uint8 and a.device == device and a.is_contiguous():
        return a
    return _dev_u8(a, device)


def bounce_hits_device(gx, gy, gvx, gvy, dt_y: float, h: float, halo: float, *, rr, is_ast=None, vis=None,
                       lo: float = -np.inf, hi: float = np.inf, device: int = 0):
    """The hit list on the device, unsorted: (int32 (k, 3) tensor of
    (offset index, a, b), k, candidate-pair count) — the input of the
    device-side bounce response (sss_collide_bounce sorts it)."""
    dev = torch.device("cuda", device)
    x, y, vx, vy = (_dev_f32(a, dev) for a in (gx, gy, gvx, gvy))
    n = x.numel()
    r = _dev_f32(rr, dev)
    ast = torch.ones(n, dtype=torch.uint8, device=dev) if is_ast is None else _dev_flags(is_ast, dev)
    vv = torch.ones(n, dtype=torch.uint8, device=dev) if vis is None else _dev_flags(vis, dev)
    ctx = _lib.context(device)
    cap = max(4096, n)
    while True:
        buf = torch.empty((cap, 3), dtype=torch.int32, device=dev)
        nh, nc = ctypes.c_int64(), ctypes.c_int64()
        with torch.cuda.device(device):
            rc = ctx.lib.sss_broadphase(ctx.ptr, x.data_ptr(), y.data_ptr(), vx.data_ptr(), vy.data_ptr(),
                                        r.data_ptr(), ast.data_ptr(), vv.data_ptr(), n, float(dt_y), float(h),
                                        float(halo), float(np.float32(lo)), float(np.float32(hi)),
                                        buf.data_ptr(), cap, ctypes.byref(nh), ctypes.byref(nc),
                                        ctypes.c_void_p(_lib.stream_handle(device)))
        if rc == _lib.SSS_ERR_CAPACITY:
            cap = int(nh.value) + 1024
            continue
        ctx.check(rc)
        break
    k = int(nh.value)
    return buf[:k], k, int(nc.value)


def bounce_hits(gx, gy, gvx, gvy, dt_y: float, h: float, halo: float, *, rr, is_ast=None, vis=None,
                lo: float = -np.inf, hi: float = np.inf, device: int = 0):
    """Colliding asteroid pairs in the stripe [lo, hi) (film_producer.py:223-317).

    Returns ((i, j) int64 host arrays or None, candidate-pair count)."""
    buf, k, nc = bounce_hits_device(gx, gy, gvx, gvy, dt_y, h, halo, rr=rr, is_ast=is_ast, vis=vis, lo=lo, hi=hi,
                                    device=device)
    if k == 0:
        return None, nc
    ctx = _lib.context(device)
    with torch.cuda.device(device):                               # (offset, a, b): the reference's order
        ctx.check(ctx.lib.sss_broadphase_order(ctx.ptr, buf.data_ptr(), k, len(gx),
                                               ctypes.c_void_p(_lib.stream_handle(device))))
    h_ = buf.cpu().numpy()
    return (h_[:, 1].astype(np.int64), h_[:, 2].astype(np.int64)), nc


class Erkennungskarte:
    """One detection GPU and its resident helper arrays (film_producer.py:166-221).

    Owns the x stripe [lo, hi): a pair belongs to it if min(x_i, x_j) lies in
    the stripe; bodies up to hi + halo are searched."""

    def __init__(self, dev: int, is_ast, lo: float, hi: float):
        self.dev = int(dev)
        self.lo = np.float32(lo)
        self.hi = np.float32(hi)
        self.g_ast = _dev_u8(is_ast, torch.device("cuda", self.dev))
        self.g_vis = None
        self.g_rr = None

    def stammdaten(self, vis, real_r) -> None:
        d = torch.device("cuda", self.dev)
        self.g_vis = _dev_u8(vis, d)
        self.g_rr = _dev_f32(real_r, d)

    def hochladen(self, outs) -> torch.Tensor:
        """One host->device transfer for a whole batch."""
        return torch.as_tensor(np.ascontiguousarray(outs)).to(torch.device("cuda", self.dev))

    def streifen(self, lo: float, hi: float) -> None:
        self.lo = np.float32(lo)
        self.hi = np.float32(hi)

    def bounce_hits(self, gx, gy, gvx, gvy, dt_y: float, h: float, halo: float):
        """((i, j) host arrays of the colliding pairs or None, candidate count)."""
        return bounce_hits(gx, gy, gvx, gvy, dt_y, h, halo, rr=self.g_rr, is_ast=self.g_ast, vis=self.g_vis,
                           lo=float(self.lo), hi=float(self.hi), device=self.dev)


def _zellschluessel(cx, cy):
    """The reference's cell hash (film_producer.py:320-321), int64 wrap-around."""
    cx = np.asarray(cx, np.int64)
    cy = np.asarray(cy, np.int64)
    with np.errstate(over="ignore"):
        return cx * np.int64(73856093) ^ cy * np.int64(19349663)


def percentile_linear(sorted_vals, q: float) -> float:
    """NumPy's default ("linear") percentile of the ascending f32 values
    `sorted_vals` (NumPy array or device tensor; NaN sorts last and makes the
    result NaN), with NumPy 2's arithmetic for f32 input, all of it in f32:
    q / 100, the virtual index (n - 1) * q, its fractional part t, and the
    interpolation a + (b - a) t, or b - (b - a)(1 - t) for t >= 1/2. Only the
    two neighbours and the last value are read (one readback from a device
    tensor)."""
    f32 = np.float32
    n = int(sorted_vals.shape[0])
    if n == 0:
        raise ValueError("percentile of an empty sample")
    vi = f32(n - 1) * (f32(q) / f32(100))
    lo = np.floor(vi)
    need = [n - 1] if vi >= n - 1 else [n - 1, int(lo), int(lo) + 1]
    if isinstance(sorted_vals, torch.Tensor):
        got = torch.stack([sorted_vals[i] for i in need]).cpu().numpy().astype(f32)
    else:
        got = np.asarray(sorted_vals)[need].astype(f32)
    if np.isnan(got[0]):
        return float("nan")
    if vi >= n - 1:
        return float(got[0])
    a, b = got[1], got[2]
    t = vi - lo
    d = b - a
    if t >= 0.5:
        return float(b - d * (f32(1) - t))
    return float(a + d * t)


def search_cell(gvx, gvy, alive, dt_y: float) -> float:
    """The broadphase cell size h = max(1e-4, 2 v95 dt) of bounce_suche
    (film_producer.py:357-359): v95 the 95th percentile of the f32 speeds
    hypot(vx, vy) of the living asteroids (device mask `alive`), the speeds
    rounded as the C library's hypotf rounds them (exact squares in f64, one
    square root), sorted on the device."""
    dev = alive.device
    vx = _dev_f32(gvx, dev).double()
    vy = _dev_f32(gvy, dev).double()
    speed = torch.sqrt(vx * vx + vy * vy).float()[alive]
    v95 = percentile_linear(torch.sort(speed).values, 95)
    return max(1e-4, 2.0 * v95 * dt_y)


def bounce_suche(det, det_pool, rows, dt_y: float, rr_max: float, anteile=None):
    """Asteroid x asteroid collisions of one sample (film_producer.py:324-379).

    One B200 is one detection card and owns the whole x range: the card
    searches (-inf, inf), so there is no stripe split and no load to balance;
    the shares come back as given (uniform when absent or of the wrong
    length), as the reference returns them for a single card. rows[0] holds
    the sample's f32 fields (x, y, vx, vy); further rows and det_pool are
    not used. The reach is the reference's: h from search_cell and a halo
    of 2h + 2 r_max. Returns (hits | None, candidate count, h, shares)."""
    n_rows = len(rows)
    shares = list(anteile) if anteile is not None and len(anteile) == n_rows else [1.0 / n_rows] * n_rows
    card = det[0]
    gx, gy, gvx, gvy = rows[0]
    alive = (card.g_ast != 0) & (card.g_vis != 0)
    if int(alive.sum()) < 2:
        return None, 0, 0.0, shares
    h = search_cell(gvx, gvy, alive, dt_y)
    card.streifen(-np.inf, np.inf)
    hits, cand = card.bounce_hits(gx, gy, gvx, gvy, dt_y, h, 2.0 * h + 2.0 * rr_max)
    return hits, cand, h, shares
