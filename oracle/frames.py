"""CPU oracle (test infrastructure only) of the server's per-sample stream
core (reference backend/server.py): display coordinates (_anzeige_koords,
:99-111), the reference box, culling by box and kill time, the density LOD
(_lod_auswahl :629-684, _dichte_filter :686-747, _index_hash :117-131) and
the u16 quantisation of build_frame (:378-537). Pinned by golden frames the
reference's own build_frame produced (tests/golden/make_golden_frames.py).

NumPy 2 promotion rules decide the precision of every step: the sample is
f32 and Python float constants are cast to f32 (comparisons, the box
offsets, the quantisation); cell weights and the bisection are f64; the
sub-cell fractions are f64 (f32 minus int32 promotes).
"""
from __future__ import annotations

import math

import numpy as np

FILM_LOG33 = float(np.log(33.0))
LOD_ZELLEN = 512
LOD_GAMMA = 0.5
LOD_MASSEN_WOLKE_AB = 200
LOD_MASSEN_ANTEIL = 0.5


def display_coords(x, y, log_zoom):
    if not log_zoom:
        return x, y
    r = np.hypot(x, y)
    sk = np.where(r > 1e-9, np.log1p(r) / (FILM_LOG33 * np.maximum(r, 1e-30)), 0.0)
    return x * sk, y * sk


def index_hash(idx):
    """SplitMix64 finalizer of the index -> [0, 1) f64."""
    h = np.asarray(idx).astype(np.uint64)
    h ^= h >> np.uint64(30)
    h *= np.uint64(0xBF58476D1CE4E5B9)
    h ^= h >> np.uint64(27)
    h *= np.uint64(0x94D049BB133111EB)
    h ^= h >> np.uint64(31)
    return (h >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def density_filter(idx, x, y, box, budget):
    if len(idx) <= budget:
        return idx
    x0, y0, spanx, spany = box
    k = LOD_ZELLEN
    cx = np.clip(((x[idx] - x0) / spanx * k).astype(np.int32), 0, k - 1)
    cy = np.clip(((y[idx] - y0) / spany * k).astype(np.int32), 0, k - 1)
    count = np.bincount(cy * k + cx, minlength=k * k)
    occ = count > 0
    weight = np.zeros(k * k)
    weight[occ] = count[occ] ** LOD_GAMMA
    lo, hi = 0.0, float(budget)
    for _ in range(40):
        s = 0.5 * (lo + hi)
        if np.minimum(count, s * weight).sum() > budget:
            hi = s
        else:
            lo = s
    goal = np.minimum(count, lo * weight)
    rate = np.zeros((k, k))
    np.divide(goal, count, out=rate.reshape(-1), where=occ)
    fx = np.clip((x[idx] - x0) / spanx * k - 0.5, 0, k - 1)
    fy = np.clip((y[idx] - y0) / spany * k - 0.5, 0, k - 1)
    ix = np.floor(fx).astype(np.int32)
    iy = np.floor(fy).astype(np.int32)
    ix1 = np.minimum(ix + 1, k - 1)
    iy1 = np.minimum(iy + 1, k - 1)
    tx = fx - ix
    ty = fy - iy
    r_p = (rate[iy, ix] * (1 - tx) * (1 - ty) + rate[iy, ix1] * tx * (1 - ty) + rate[iy1, ix] * (1 - tx) * ty
           + rate[iy1, ix1] * tx * ty)
    return idx[index_hash(idx) < r_p]


def lod_select(sel, x, y, box, budget, is_ast, injected):
    if len(sel) <= budget:
        return sel
    ast = is_ast[sel]
    massive = sel[~ast]
    rest = budget - len(massive)
    if rest <= 0:
        if len(massive) > LOD_MASSEN_WOLKE_AB and len(sel) > len(massive):
            m_budget = max(1, int(budget * LOD_MASSEN_ANTEIL))
            parts = [density_filter(massive, x, y, box, m_budget)]
            rest = budget - len(parts[0])
            a_sel = sel[ast]
            if rest > 0 and len(a_sel):
                parts.append(density_filter(a_sel, x, y, box, rest))
            return np.sort(np.concatenate(parts))
        return sel[~ast]
    a_sel = sel[ast]
    inj = injected[a_sel]
    parts = [massive]
    for cand in (a_sel[~inj], a_sel[inj]):
        if rest <= 0 or not len(cand):
            continue
        kept = density_filter(cand, x, y, box, rest)
        parts.append(kept)
        rest -= len(kept)
    return np.sort(np.concatenate(parts))


def make_box(qxs, qys, view):
    cx, cy, hw, hh = (float(v) for v in view)      # Python floats, as the session's view tuple
    if hw <= 0 or hh <= 0:
        bx0, bx1 = float(qxs.min()), float(qxs.max())
        by0, by1 = float(qys.min()), float(qys.max())
        mx = 0.05 * max(bx1 - bx0, 1e-6)
        my = 0.05 * max(by1 - by0, 1e-6)
        return (bx0 - mx, by0 - my, max(bx1 - bx0 + 2 * mx, 1e-6), max(by1 - by0 + 2 * my, 1e-6))
    return (cx - 2 * hw, cy - 2 * hh, max(4 * hw, 1e-6), max(4 * hh, 1e-6))


def sample_frame(x, y, alive, is_ast, injected, box, log_zoom, budget):
    """(sel u32, qx u16, qy u16) of one f32 sample inside box."""
    qxs, qys = display_coords(np.asarray(x, np.float32), np.asarray(y, np.float32), log_zoom)
    box = tuple(float(v) for v in box)             # Python floats: weak scalars, cast to f32 against f32 arrays
    x0, y0, spanx, spany = box
    sel = np.flatnonzero(alive & (qxs >= x0) & (qxs <= x0 + spanx) & (qys >= y0) & (qys <= y0 + spany))
    sel = lod_select(sel, qxs, qys, box, budget, is_ast, injected)
    qx = np.clip((qxs[sel] - x0) / spanx * 65535.0, 0, 65535).astype("<u2")
    qy = np.clip((qys[sel] - y0) / spany * 65535.0, 0, 65535).astype("<u2")
    return sel.astype("<u4"), qx, qy


def lod_budget(lod_budget_setting, bandwidth):
    """The points a sample may carry (build_frame's lod_max)."""
    return lod_budget_setting or min(120_000, max(20000, int(bandwidth * 0.7 / 20.0 / 8.0)))


__all__ = ["display_coords", "index_hash", "density_filter", "lod_select", "make_box", "sample_frame",
           "lod_budget", "math"]
