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


def _f32_bits(x):
    return np.asarray(x, np.float32).view(np.int32)


def _f32_of(bits):
    return np.asarray(bits, np.int32).view(np.float32)


_LN2_HI = _f32_of(0x3F317180)
_LN2_LO = _f32_of(0x3717F7D1)
_LOG1P_R = [_f32_of(b) for b in (0x3F2AAAAB, 0x3ECCCCCD, 0x3E924925, 0x3E638E29, 0x3E3A3325, 0x3E1CD04F,
                                  0x3E178897)]


def log1p_f32(x):
    """log(1 + x) for f32 x >= 0, every operation rounded to f32, by the
    published reduction method of fdlibm's log1pf (Sun Microsystems, 1993),
    which is the f32 log1p of the C library (glibc up to 2.40) that NumPy
    calls for float32 log1p where it dispatches no SIMD kernel:
    1 + x = 2^k (1 + f) with sqrt(2)/2 <= 1 + f < sqrt(2) and a correction
    c for the rounding of 1 + x; s = f / (2 + f);
    log(1 + f) = f - (hfsq - s (hfsq + R(s^2))), hfsq = f^2 / 2, R a
    degree-7 minimax polynomial; k ln 2 in two parts. Checked bit for bit
    against the C library's log1pf on every f32 in [2^-31, 2^22)."""
    F = np.float32
    x = np.asarray(x, np.float32)
    hx = _f32_bits(x)
    out = np.full(x.shape, np.nan, np.float32)
    tiny = (hx >= 0) & (hx < 0x31000000)                               # x < 2^-29
    xt = x[tiny]
    out[tiny] = np.where(hx[tiny] < 0x24800000, xt, xt - xt * xt * F(0.5))
    near = (hx >= 0x31000000) & (hx < 0x3ED413D7)                      # 2^-29 <= x < 0.41422: k = 0
    far = (hx >= 0x3ED413D7) & (hx < 0x7F800000)
    big = hx >= 0x7F800000                                             # inf, nan
    out[big] = x[big] + x[big]
    xf, hf = x[far], hx[far]
    small_u = hf < 0x5A000000
    u = np.where(small_u, xf + F(1.0), xf).astype(np.float32)
    hu = _f32_bits(u)
    k = (hu >> 23) - 127
    c = np.where(k > 0, F(1.0) - (u - xf), xf - (u - F(1.0))).astype(np.float32)
    c = np.where(small_u, c / u, F(0.0)).astype(np.float32)
    hu = hu & 0x007FFFFF
    low = hu < 0x3504F7
    u = np.where(low, _f32_of(hu | 0x3F800000), _f32_of(hu | 0x3F000000))
    k = np.where(low, k, k + 1)
    hu = np.where(low, hu, (0x00800000 - hu) >> 2)

    def finish(f, k, c, hu):
        # the k = 0 forms drop the correction c, also where k comes out 0 after the reduction
        kf = k.astype(np.float32)
        k0 = k == 0
        hfsq = F(0.5) * f * f
        res = np.empty(f.shape, np.float32)
        e = (hu == 0) & (f == 0)
        res[e] = np.where(k0[e], F(0.0), kf[e] * _LN2_HI + (c[e] + kf[e] * _LN2_LO))
        t = (hu == 0) & (f != 0)                                       # |f| < 2^-20
        ft = f[t]
        R = hfsq[t] * (F(1.0) - F(0.66666666666666666) * ft)
        res[t] = np.where(k0[t], ft - R, kf[t] * _LN2_HI - ((R - (kf[t] * _LN2_LO + c[t])) - ft))
        g = hu != 0
        fg, hq = f[g], hfsq[g]
        s = fg / (F(2.0) + fg)
        z = s * s
        R = z * (_LOG1P_R[0] + z * (_LOG1P_R[1] + z * (_LOG1P_R[2] + z * (_LOG1P_R[3] + z * (
            _LOG1P_R[4] + z * (_LOG1P_R[5] + z * _LOG1P_R[6]))))))
        res[g] = np.where(k0[g], fg - (hq - s * (hq + R)),
                          kf[g] * _LN2_HI - ((hq - (s * (hq + R) + (kf[g] * _LN2_LO + c[g]))) - fg))
        return res

    xn = x[near]
    out[near] = finish(xn, np.zeros(xn.shape, np.int32), np.zeros(xn.shape, np.float32),
                       np.ones(xn.shape, np.int32))
    out[far] = finish((u - F(1.0)).astype(np.float32), k, c, hu)
    return out


def hypot_f32(x, y):
    """f32 hypot correctly rounded: the squares of f32 values are exact in
    f64, their sum is rounded once, the f64 square root once more, then the
    result to f32 (what the C library's hypotf returns for finite input)."""
    xd = np.asarray(x, np.float32).astype(np.float64)
    yd = np.asarray(y, np.float32).astype(np.float64)
    r = np.sqrt(xd * xd + yd * yd).astype(np.float32)
    inf = np.isinf(xd) | np.isinf(yd)
    return np.where(inf, np.float32(np.inf), r)


def display_coords(x, y, log_zoom):
    """_anzeige_koords (server.py:99-111) with NumPy's float32 hypot and
    log1p taken as the C library computes them (log1p_f32, hypot_f32).
    NumPy on a CPU with AVX512_SKX dispatches float32 log1p to a SIMD
    kernel that differs from the C library in the last bit or two for
    about 10 % of the inputs; the golden log-zoom frame is written with
    that dispatch switched off (tests/golden/make_golden_frames.py)."""
    if not log_zoom:
        return x, y
    r = hypot_f32(x, y)
    sk = np.where(r > 1e-9, log1p_f32(r) / (FILM_LOG33 * np.maximum(r, 1e-30)), 0.0)
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
