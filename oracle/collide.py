"""CPU oracle (test infrastructure only) of the reference's collision
response in the film producer: the merge sweep of the massive bodies
(`analyze_merge`, backend/film_producer.py:707-779), the merge application
(`apply_merges`, :781-861) and the bounce response (`bounce_deltas`,
:916-1019; hit order from `Erkennungskarte._hits`, :223-321).

The reference evaluates the sweep with CuPy element-wise f32 operations
(one rounding per operation, no fused multiply-add) and the bounce response
with NumPy f64 on values upcast from the f32 snapshot; NumPy reproduces both
operation for operation. Its closures live inside producer_main and cannot
be imported, so this restatement follows their lines (parity against the
reference's own outputs is unpinned; the GPU kernels are checked against it
bit for bit on integer results and to 1e-12 on f64 results).
"""
from __future__ import annotations

import numpy as np

BOUNCE_E = 0.6            # restitution (film_producer.py:47)
G_AU = 4.0 * np.pi * np.pi


def np_pairwise_sum(a):
    """NumPy's pairwise summation of a contiguous f64 vector (the order
    ndarray.sum uses; blocks of 128, eight interleaved partial sums)."""
    a = np.asarray(a, np.float64)
    n = len(a)
    if n < 8:
        r = 0.0
        for v in a:
            r += v
        return r
    if n <= 128:
        r = [a[j] for j in range(8)]
        i = 8
        while i < n - (n % 8):
            for j in range(8):
                r[j] += a[i + j]
            i += 8
        res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]))
        while i < n:
            res += a[i]
            i += 1
        return res
    n2 = n // 2
    n2 -= n2 % 8
    return np_pairwise_sum(a[:n2]) + np_pairwise_sum(a[n2:])


def _seg_hit(p0x, p0y, p1x, p1y, cx, cy, rsum2):
    """Segment p0 -> p1 against the spheres (cx, cy, rsum): f32, one
    rounding per operation (film_producer.py:729-748)."""
    f32 = np.float32
    ssx = (p1x - p0x)[None, :]
    ssy = (p1y - p0y)[None, :]
    seg2 = ssx * ssx + ssy * ssy
    den = np.where(seg2 > 0, seg2, f32(1.0))
    tt = ((cx - p0x[None, :]) * ssx + (cy - p0y[None, :]) * ssy) / den
    tt = np.clip(tt, f32(0.0), f32(1.0))
    ddx = p0x[None, :] + tt * ssx - cx
    ddy = p0y[None, :] + tt * ssy - cy
    return ddx * ddx + ddy * ddy <= rsum2, tt


def merge_sweep(gx, gy, gvx, gvy, px, py, rr32, vis, is_ast, mass, m_idx, dt_y, G=G_AU):
    """Merge candidates and runaways of one sample (film_producer.py:707-779).

    gx..gvy: f32 snapshot of this sample; px, py: f32 positions of the
    previous sample (the current ones on the first call); rr32: f32 contact
    radii; vis, is_ast: flags; mass: f64; m_idx: original indices of the
    massive bodies (ascending). Returns (pairs [(massive, j, frac)], runaways
    int64 array or None)."""
    f32 = np.float32
    gx, gy, gvx, gvy, px, py = (np.asarray(a, f32) for a in (gx, gy, gvx, gvy, px, py))
    rr32 = np.asarray(rr32, f32)
    vis = np.asarray(vis)
    mass = np.asarray(mass, np.float64)
    m_idx = np.asarray(m_idx, np.int64)
    m_alive = m_idx[(vis[m_idx] != 0) & (mass[m_idx] > 0)]
    pairs, runaway = [], None
    if len(m_alive):
        cx = gx[m_alive][:, None]
        cy = gy[m_alive][:, None]
        rsum = rr32[m_alive][:, None] + rr32[None, :]
        rsum2 = rsum * rsum
        alive = vis != 0
        g_dt = f32(dt_y)
        hit_a, tt_a = _seg_hit(px, py, gx, gy, cx, cy, rsum2)
        hit_b, tt_b = _seg_hit(gx, gy, gx + gvx * g_dt, gy + gvy * g_dt, cx, cy, rsum2)
        hit2d = (hit_a | hit_b) & alive[None, :]
        frac2d = np.where(hit_a, tt_a - f32(1.0), tt_b)
        hit2d[np.arange(len(m_alive)), m_alive] = False
        rows, cols = np.nonzero(hit2d)
        pairs = [(int(m_alive[r]), int(c), float(frac2d[r, c])) for r, c in zip(rows, cols)]
        mw = mass[m_alive]
        msum = float(np_pairwise_sum(mw))
        if msum > 0:
            bx = float(np_pairwise_sum(gx[m_alive].astype(np.float64) * mw) / msum)
            by = float(np_pairwise_sum(gy[m_alive].astype(np.float64) * mw) / msum)
            r = np.maximum(np.hypot(gx - f32(bx), gy - f32(by)), f32(1e-6))
            v2 = gvx * gvx + gvy * gvy
            vesc2 = f32(2.0 * G * msum) / r
            run = (v2 > f32(9.0) * vesc2) & (np.asarray(is_ast) != 0) & alive
            ridx = np.flatnonzero(run)
            if ridx.size:
                runaway = ridx.astype(np.int64)
    return pairs, runaway


def sweep_barycentre(gx, gy, mass, m_alive):
    """(bx, by, msum) as merge_sweep forms them (f64)."""
    mw = np.asarray(mass, np.float64)[m_alive]
    msum = float(np_pairwise_sum(mw))
    bx = float(np_pairwise_sum(np.asarray(gx, np.float32)[m_alive].astype(np.float64) * mw) / msum)
    by = float(np_pairwise_sum(np.asarray(gy, np.float32)[m_alive].astype(np.float64) * mw) / msum)
    return bx, by, msum


def bounce_filter(hi, hj):
    """At most one hit per body per sample, in hit order (:928-943)."""
    used = set()
    keep = []
    for t, (a, b) in enumerate(zip(hi, hj)):
        a, b = int(a), int(b)
        if a in used or b in used:
            continue
        used.add(a)
        used.add(b)
        keep.append(t)
    return np.asarray(keep, np.int64)


def bounce_deltas(x, y, vx, vy, real_r, mass, hi, hj, dt_y, e=BOUNCE_E):
    """Impulse and overlap push of the kept hits (:916-1019). x..vy f32
    snapshot arrays, real_r and mass f64; hi, hj the hit list in order.
    Returns None or (hi, hj, touched int64 ascending, deltas (m, 4) f64
    [dx, dy, dvx, dvy])."""
    x, y, vx, vy = (np.asarray(a, np.float32) for a in (x, y, vx, vy))
    real_r = np.asarray(real_r, np.float64)
    mass = np.asarray(mass, np.float64)
    n = len(x)
    keep = bounce_filter(hi, hj)
    if not len(keep):
        return None
    hi = np.asarray(hi)[keep].astype(np.int64)
    hj = np.asarray(hj)[keep].astype(np.int64)
    dpx = x[hj].astype(np.float64) - x[hi].astype(np.float64)
    dpy = y[hj].astype(np.float64) - y[hi].astype(np.float64)
    dvx = vx[hj].astype(np.float64) - vx[hi].astype(np.float64)
    dvy = vy[hj].astype(np.float64) - vy[hi].astype(np.float64)
    dv2 = dvx * dvx + dvy * dvy
    touch = real_r[hi] + real_r[hj]
    c_ = dpx * dpx + dpy * dpy - touch * touch
    b_ = 2.0 * (dpx * dvx + dpy * dvy)
    disc = b_ * b_ - 4.0 * dv2 * c_
    sq = np.sqrt(np.maximum(disc, 0.0))
    with np.errstate(divide="ignore", invalid="ignore"):
        t_enter = (-b_ - sq) / (2.0 * np.where(dv2 > 0, dv2, 1.0))
    t_c = np.where(c_ < 0.0, 0.0, np.clip(np.nan_to_num(t_enter), -dt_y, dt_y))
    valid = (c_ < 0.0) | (disc >= -(touch * touch) * 0.01)
    ncx = dpx + dvx * t_c
    ncy = dpy + dvy * t_c
    dist = np.hypot(ncx, ncy)
    dist = np.where(dist > 1e-30, dist, 1.0)
    nx = ncx / dist
    ny = ncy / dist
    vrel = dvx * nx + dvy * ny
    act = valid & (vrel < 0)
    if not act.any():
        return None
    hi, hj, nx, ny, vrel = hi[act], hj[act], nx[act], ny[act], vrel[act]
    mi, mj = mass[hi], mass[hj]
    with np.errstate(divide="ignore", invalid="ignore"):
        imp = -(1.0 + e) * vrel / (1.0 / mi + 1.0 / mj)
    imp = np.nan_to_num(imp)
    ddx, ddy, ddvx, ddvy = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    err = np.seterr(divide="ignore", invalid="ignore")      # massless pairs give NaN, as in the reference
    ddvx[hi] -= imp * nx / mi
    ddvy[hi] -= imp * ny / mi
    ddvx[hj] += imp * nx / mj
    ddvy[hj] += imp * ny / mj
    pdx = x[hj].astype(np.float64) - x[hi].astype(np.float64)
    pdy = y[hj].astype(np.float64) - y[hi].astype(np.float64)
    pdist = np.hypot(pdx, pdy)
    touch = real_r[hi] + real_r[hj]
    overlap = touch - pdist
    ol = (overlap > 0) & (pdist > 1e-30)
    if ol.any():
        oi, oj = hi[ol], hj[ol]
        pnx = pdx[ol] / pdist[ol]
        pny = pdy[ol] / pdist[ol]
        mges = mass[oi] + mass[oj]
        wa = mass[oj] / mges
        wb = mass[oi] / mges
        shift = overlap[ol] * 1.1
        ddx[oi] -= pnx * shift * wa
        ddy[oi] -= pny * shift * wa
        ddx[oj] += pnx * shift * wb
        ddy[oj] += pny * shift * wb
    np.seterr(**err)
    touched = np.unique(np.concatenate([hi, hj]))
    deltas = np.stack([ddx[touched], ddy[touched], ddvx[touched], ddvy[touched]], axis=1)
    return hi, hj, touched.astype(np.int64), deltas


def apply_merges(sample, n, pairs, runaways, mass, vis, real_r, is_ast, is_star_bh, k_ev=0, contact=None,
                 shatter=True, G=G_AU):
    """Sequential application of the merge candidates and runaways
    (:781-861). sample: f32 (4n,) [x|y|vx|vy]; mass, vis, real_r are updated
    in place. contact: dict body -> fine-loop contact time (consumed).
    Returns (events, body_states, deactivated, shatter_pair):
    events (a, b, new_mass, kind, frac, x, y) with kind 0 merge, 2 runaway;
    body_states (a, x, y, vx, vy, m, r) to apply; shatter_pair (a, b, frac)
    or None — when set, processing stopped there as in the reference."""
    sx, sy = sample[0:n], sample[n:2 * n]
    svx, svy = sample[2 * n:3 * n], sample[3 * n:4 * n]
    events, states, deact = [], [], []
    contact = {} if contact is None else contact
    for mi, j, frac in pairs:
        tk = contact.pop(j, None)
        if tk is not None:
            f_kern = tk - (k_ev + 1)
            if -1.0 <= f_kern <= 1.0:
                frac = f_kern
        if (shatter and not is_ast[mi] and not is_ast[j] and not is_star_bh[mi] and not is_star_bh[j]
                and vis[mi] and vis[j] and mass[mi] > 0 and mass[j] > 0):
            v_imp = float(np.hypot(sample[2 * n + j] - sample[2 * n + mi], sample[3 * n + j] - sample[3 * n + mi]))
            touch = max(1e-12, real_r[mi] + real_r[j])
            v_esc = float(np.sqrt(2.0 * G * (mass[mi] + mass[j]) / touch))
            if v_imp >= 1.5 * v_esc:
                return events, states, deact, (int(mi), int(j), frac)
        if not vis[mi] or not vis[j] or mass[mi] <= 0:
            continue
        a, b = (mi, j) if mass[mi] >= mass[j] else (j, mi)
        m_a, m_b = mass[a], mass[b]
        m_ges = m_a + m_b
        if m_ges <= 0:
            continue
        nx = (sx[a] * m_a + sx[b] * m_b) / m_ges
        ny = (sy[a] * m_a + sy[b] * m_b) / m_ges
        nvx = (svx[a] * m_a + svx[b] * m_b) / m_ges
        nvy = (svy[a] * m_a + svy[b] * m_b) / m_ges
        mass[a] = m_ges
        mass[b] = 0.0
        vis[b] = 0
        real_r[a] = (real_r[a] ** 3 + real_r[b] ** 3) ** (1.0 / 3.0)
        states.append((int(a), float(nx), float(ny), float(nvx), float(nvy), float(m_ges), float(real_r[a])))
        deact.append(int(b))
        events.append((int(a), int(b), float(m_ges), 0, float(frac), float(nx), float(ny)))
    if runaways is not None:
        for j in runaways:
            j = int(j)
            if not vis[j]:
                continue
            mass[j] = 0.0
            vis[j] = 0
            deact.append(j)
            events.append((0xFFFFFFFF, j, 0.0, 2, 0.0, float(sx[j]), float(sy[j])))
    return events, states, deact, None


def _frag_uniform(seed, a, b, k, j):
    """SplitMix64 of (seed, a, b, fragment k, draw j) -> [0, 1) f64, the
    device generator of sss_collide_fragment."""
    M = (1 << 64) - 1
    h = (seed ^ ((a * 0x9E3779B97F4A7C15) & M) ^ ((b * 0xC2B2AE3D27D4EB4F) & M)) & M
    h = (h + (2 * k + j + 1) * 0xD6E8FEB86659FD93) & M
    h ^= h >> 30
    h = (h * 0xBF58476D1CE4E5B9) & M
    h ^= h >> 27
    h = (h * 0x94D049BB133111EB) & M
    h ^= h >> 31
    return float(h >> 11) * 2.0 ** -53


def fragment_events(x, y, vx, vy, real_r, mass, pairs, G, factor, seed, n_frag=5):
    """Fragmentation of fast impacts among the active bounce pairs, in f64
    (the construction of the reference client's shatter(), index.html:
    7705-7745, with a seeded generator): [(a, b, fragments (n_frag, 6) of
    x, y, vx, vy, m, r)] in pair order."""
    out = []
    if factor <= 0:
        return out
    x, y, vx, vy = (np.asarray(v, np.float32) for v in (x, y, vx, vy))
    rr = np.asarray(real_r, np.float64)
    mass = np.asarray(mass, np.float64)
    for a, b in pairs:
        a, b = int(a), int(b)
        ma, mb = mass[a], mass[b]
        mt = ma + mb
        if not mt > 0.0:
            continue
        dvx = float(vx[b]) - float(vx[a])
        dvy = float(vy[b]) - float(vy[a])
        v_imp = np.sqrt(dvx * dvx + dvy * dvy)
        touch = max(rr[a] + rr[b], 1e-12)
        if not v_imp >= factor * np.sqrt(2.0 * G * mt / touch):
            continue
        cx = (ma * float(x[a]) + mb * float(x[b])) / mt
        cy = (ma * float(y[a]) + mb * float(y[b])) / mt
        cvx = (ma * float(vx[a]) + mb * float(vx[b])) / mt
        cvy = (ma * float(vy[a]) + mb * float(vy[b])) / mt
        ring = rr[a] + rr[b]
        rf = np.cbrt((rr[a] ** 3 + rr[b] ** 3) / n_frag)
        ang = [2.0 * np.pi * k / n_frag + (_frag_uniform(seed, a, b, k, 0) - 0.5) * 0.6 for k in range(n_frag)]
        spd = [v_imp * (0.25 + 0.35 * _frag_uniform(seed, a, b, k, 1)) for k in range(n_frag)]
        mx = sum(np.cos(t) * s for t, s in zip(ang, spd)) / n_frag
        my = sum(np.sin(t) * s for t, s in zip(ang, spd)) / n_frag
        f = np.empty((n_frag, 6))
        for k in range(n_frag):
            th = 2.0 * np.pi * k / n_frag
            f[k] = (cx + np.cos(th) * ring, cy + np.sin(th) * ring, cvx + (np.cos(ang[k]) * spd[k] - mx),
                    cvy + (np.sin(ang[k]) * spd[k] - my), mt / n_frag, rf)
        out.append((a, b, f))
    return out
