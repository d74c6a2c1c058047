"""Asteroid x asteroid collision broadphase on one B200.

Drop-in for the detection layer of the reference's backend/film_producer.py
(`Erkennungskarte`, `_zellschluessel`, `bounce_suche`, `_streifengrenzen`,
`NACHBARN`, `CHUNK`). The pair search runs in libsss (`sss_broadphase`); the
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
LAST_ALPHA = 0.35                                     # film_producer.py:410


def _dev_f32(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float32).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(device)


def _dev_u8(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return (a != 0).to(device=device, dtype=torch.uint8).contiguous()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a) != 0, dtype=np.uint8)).to(device)


def bounce_hits_device(gx, gy, gvx, gvy, dt_y: float, h: float, halo: float, *, rr, is_ast=None, vis=None,
                       lo: float = -np.inf, hi: float = np.inf, device: int = 0):
    """The hit list on the device, unsorted: (int32 (k, 3) tensor of
    (offset index, a, b), k, candidate-pair count) — the input of the
    device-side bounce response (sss_collide_bounce sorts it)."""
    dev = torch.device("cuda", device)
    x, y, vx, vy = (_dev_f32(a, dev) for a in (gx, gy, gvx, gvy))
    n = x.numel()
    r = _dev_f32(rr, dev)
    ast = torch.ones(n, dtype=torch.uint8, device=dev) if is_ast is None else _dev_u8(is_ast, dev)
    vv = torch.ones(n, dtype=torch.uint8, device=dev) if vis is None else _dev_u8(vis, dev)
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


def _streifengrenzen(gx_lebt, anteile):
    """x stripes holding the given shares of the living asteroids
    (film_producer.py:382-405); the outer bounds are infinite."""
    if len(anteile) < 2:
        return [(-np.inf, np.inf)]
    q, lauf = [], 0.0
    for a in anteile[:-1]:
        lauf += a
        q.append(100.0 * lauf)
    g = gx_lebt.cpu().numpy() if isinstance(gx_lebt, torch.Tensor) else np.asarray(gx_lebt)
    schnitte = [float(v) for v in np.percentile(g, q)]
    kanten = [-np.inf, *schnitte, np.inf]
    return list(zip(kanten[:-1], kanten[1:]))


LAST_MIN_ANTEIL = 0.05                                # film_producer.py:415


def _lastanteile(anteile, last):
    """Stripe shares for the next sample from the measured candidate counts
    (film_producer.py:418-479): each share is multiplied by
    (fair share / measured share) ** LAST_ALPHA, renormalised, and shares
    below LAST_MIN_ANTEIL are pinned there while the rest share the
    remaining room (uniform shares if that room is gone)."""
    n = len(anteile)
    if n < 2:
        return list(anteile)
    ges = float(sum(last))
    if ges <= 0 or min(last) < 0:
        return list(anteile)
    neu = [max(anteile[i] * ((1.0 / n) / max(last[i] / ges, 1e-9)) ** LAST_ALPHA, 1e-6) for i in range(n)]
    summe = sum(neu)
    neu = [a / summe for a in neu]
    klein = [a < LAST_MIN_ANTEIL for a in neu]
    if any(klein):
        platz = 1.0 - LAST_MIN_ANTEIL * sum(klein)
        rest = sum(a for a, k in zip(neu, klein) if not k)
        if platz <= 0 or rest <= 0:
            return [1.0 / n] * n
        neu = [LAST_MIN_ANTEIL if k else a / rest * platz for a, k in zip(neu, klein)]
    return neu


def bounce_suche(det, det_pool, rows, dt_y: float, rr_max: float, anteile=None):
    """Asteroid x asteroid collisions over the detection cards
    (film_producer.py:324-379): h from the 95th speed percentile, halo
    2h + 2 r_max, one stripe per card. Returns (hits | None, candidates,
    h, new shares)."""
    gx, gy, gvx, gvy = rows[0]
    if anteile is None or len(anteile) != len(rows):
        anteile = [1.0 / len(rows)] * len(rows)
    k0 = det[0]
    dev = torch.device("cuda", k0.dev)
    lebt = torch.nonzero((k0.g_ast != 0) & (k0.g_vis != 0)).flatten()
    if lebt.numel() < 2:
        return None, 0, 0.0, anteile
    vx_t, vy_t = _dev_f32(gvx, dev), _dev_f32(gvy, dev)
    speed = torch.hypot(vx_t[lebt], vy_t[lebt]).double()
    v95 = float(torch.quantile(speed, 0.95))
    grenzen = _streifengrenzen(_dev_f32(gx, dev)[lebt], anteile)
    h = max(1e-4, 2.0 * v95 * dt_y)
    halo = 2.0 * h + 2.0 * rr_max
    for karte, (lo, hi) in zip(det, grenzen):
        karte.streifen(lo, hi)
    teile = [karte.bounce_hits(*row, dt_y, h, halo) for karte, row in zip(det[:len(rows)], rows)]
    hits = [t for t, _ in teile if t is not None]
    je_karte = [kand for _, kand in teile]
    neu = _lastanteile(anteile, je_karte)
    if not hits:
        return None, sum(je_karte), h, neu
    return ((np.concatenate([t[0] for t in hits]), np.concatenate([t[1] for t in hits])),
            sum(je_karte), h, neu)
