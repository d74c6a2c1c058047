"""Oracle for the collision broadphase (TEST INFRASTRUCTURE ONLY).

NumPy restatement of `Erkennungskarte._hits` and `_zellschluessel`
(reference backend/film_producer.py:223-321): alive mask in f32, cells
floor(f64(x)/h), int64 hash with wrap-around, stable sort, equal-key ranges
for the five neighbour offsets, keep rule a < b / a != b, f32 closest
approach over [-dt, dt] (each operation rounded separately, as NumPy does),
ownership min(x_a, x_b) < hi, f64 recheck. Returns the pairs in the
reference's order and the candidate count.
"""
from __future__ import annotations

import numpy as np

NACHBARN = ((0, 0), (1, 0), (0, 1), (1, 1), (1, -1))


def cell_key(cx, cy):
    with np.errstate(over="ignore"):
        return cx * np.int64(73856093) ^ cy * np.int64(19349663)


def _ccd(dpx, dpy, dvx, dvy, rsum, dt, one):
    dv2 = dvx * dvx + dvy * dvy
    tmin = np.clip(-(dpx * dvx + dpy * dvy) / np.where(dv2 > 0, dv2, one), -dt, dt)
    cxm = dpx + dvx * tmin
    cym = dpy + dvy * tmin
    return cxm * cxm + cym * cym <= rsum * rsum


def hits(gx, gy, gvx, gvy, rr, dt_y, h, halo, is_ast=None, vis=None, lo=-np.inf, hi=np.inf):
    gx, gy, gvx, gvy, rr = (np.asarray(a, np.float32) for a in (gx, gy, gvx, gvy, rr))
    n = len(gx)
    ast = np.ones(n, bool) if is_ast is None else np.asarray(is_ast) != 0
    vv = np.ones(n, bool) if vis is None else np.asarray(vis) != 0
    lo32, hi32 = np.float32(lo), np.float32(hi)
    alive = ast & vv & (gx >= lo32) & (gx < hi32 + np.float32(halo))
    ai = np.flatnonzero(alive)
    if ai.size < 2:
        return None, 0
    ix = np.floor(gx[ai].astype(np.float64) / h).astype(np.int64)
    iy = np.floor(gy[ai].astype(np.float64) / h).astype(np.int64)
    key = cell_key(ix, iy)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    f32 = np.float32
    out_i, out_j, cand = [], [], 0
    for ox, oy in NACHBARN:
        k2 = cell_key(ix + ox, iy + oy)
        lo_r = np.searchsorted(ks, k2, side="left")
        hi_r = np.searchsorted(ks, k2, side="right")
        lens = hi_r - lo_r
        tot = int(lens.sum())
        cand += tot
        if tot == 0:
            continue
        rows = np.repeat(np.arange(len(ai)), lens)
        starts = np.cumsum(lens) - lens
        cols = np.arange(tot) - starts[rows] + lo_r[rows]
        a = ai[rows]
        b = ai[order[cols]]
        keep = (a < b) if (ox == 0 and oy == 0) else (a != b)
        a, b = a[keep], b[keep]
        sel = _ccd(gx[b] - gx[a], gy[b] - gy[a], gvx[b] - gvx[a], gvy[b] - gvy[a],
                   rr[a] + rr[b] + f32(1e-6), f32(dt_y), f32(1.0))
        out_i.append(a[sel])
        out_j.append(b[sel])
    ci = np.concatenate(out_i)
    cj = np.concatenate(out_j)
    own = np.minimum(gx[ci], gx[cj]) < hi32
    ci, cj = ci[own], cj[own]
    d = np.float64
    sel = _ccd(gx[cj].astype(d) - gx[ci].astype(d), gy[cj].astype(d) - gy[ci].astype(d),
               gvx[cj].astype(d) - gvx[ci].astype(d), gvy[cj].astype(d) - gvy[ci].astype(d),
               rr[ci].astype(d) + rr[cj].astype(d), dt_y, 1.0)
    if not sel.any():
        return None, cand
    return (ci[sel], cj[sel]), cand


def hits_c(gx, gy, gvx, gvy, rr, dt_y, h, halo, is_ast=None, vis=None, lo=-np.inf, hi=np.inf, threads=None):
    """The same pair list from the C restatement (oracle/broadphase.c),
    multithreaded, for scenes the NumPy form takes minutes on."""
    import ctypes
    import os
    from . import build as _build
    L = ctypes.CDLL(_build.build())
    f = L.oracle_broadphase_hits
    f.restype = ctypes.c_int64
    vp = ctypes.c_void_p
    f.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                  ctypes.c_float, ctypes.c_float, vp, vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                  ctypes.c_int]
    arrs = [np.ascontiguousarray(a, np.float32) for a in (gx, gy, gvx, gvy, rr)]
    n = len(arrs[0])
    ast = None if is_ast is None else np.ascontiguousarray(np.asarray(is_ast) != 0, np.uint8)
    vv = None if vis is None else np.ascontiguousarray(np.asarray(vis) != 0, np.uint8)
    nthreads = threads or int(os.environ.get("SSS_ORACLE_THREADS", os.cpu_count() or 1))
    cap = max(1024, n)
    while True:
        oi = np.empty(cap, np.int64)
        oj = np.empty(cap, np.int64)
        nc = ctypes.c_int64()
        k = f(*(a.ctypes.data for a in arrs), None if ast is None else ast.ctypes.data,
              None if vv is None else vv.ctypes.data, n, float(dt_y), float(h), float(halo),
              float(np.float32(lo)), float(np.float32(hi)), oi.ctypes.data, oj.ctypes.data, cap, ctypes.byref(nc),
              nthreads)
        if k < 0:
            raise MemoryError("oracle_broadphase_hits: allocation failed")
        if k <= cap:
            break
        cap = int(k)
    if k == 0:
        return None, int(nc.value)
    return (oi[:k], oj[:k]), int(nc.value)
