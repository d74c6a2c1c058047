"""Oracle for the few-massive-body integrator (TEST INFRASTRUCTURE ONLY).

* `frame_launch`: a CPU restatement of one launch of the reference's
  `frame_kernel` (backend/nbody_kernel.py:97-560) on one device: initial
  accelerations (:151-216), K raster samples (:233-558), each a loop of
  hierarchical substeps dtH (:245-537): dtH from massive pairs (:247-275),
  hot classification (:283-301), three Yoshida velocity-Verlet stages for
  calm asteroids and massive bodies with asteroid back-reaction (:314-401),
  the private adaptive fine loop of hot asteroids against linearly
  interpolated massive positions with contact detection and sub-samples
  (:416-535), and the f32 snapshots (:540-557). Vectorised over asteroids;
  the hot fine loop is scalar.
* `reference_advance`: restatement of the reference's own NumPy oracle
  (backend/test_kernel.py:16-81): every body on one adaptive step
  (massive pairs and asteroid x massive pairs lower dt), Yoshida.

Bodies are given per dimension (x[d], v[d]) so 2-D and 3-D share the code.
"""
from __future__ import annotations

import numpy as np

G_AU = 4 * np.pi * np.pi                                  # nbody_kernel.py:60
SOFTENING = 1e-6                                          # :61
MAX_SUB_DT_YEARS = 0.5 / 365.25                           # :62
MAX_SUB_STEPS_PER_FRAME = 100_000                         # :63
YOSHIDA_W1 = 1.0 / (2.0 - 2.0 ** (1.0 / 3.0))             # :64
YOSHIDA_W0 = -(2.0 ** (1.0 / 3.0)) / (2.0 - 2.0 ** (1.0 / 3.0))  # :65


def _pair_force(dxs, soft, G):
    r2 = sum(d * d for d in dxs) + soft
    return G / (r2 * np.sqrt(r2))


class FrameState:
    """Asteroid (a*) and massive (m*) arrays, float64; x/v are (dim, n)."""

    def __init__(self, ax, av, am, avis, arad, mx, mv, mm, mvis, mrad):
        self.ax, self.av = np.array(ax, float), np.array(av, float)
        self.am = np.array(am, float)
        self.avis = np.array(avis, bool)
        self.arad = np.array(arad, float)
        self.mx, self.mv = np.array(mx, float), np.array(mv, float)
        self.mm = np.array(mm, float)
        self.mvis = np.array(mvis, bool)
        self.mrad = np.array(mrad, float)

    @property
    def dim(self):
        return self.ax.shape[0]


def _ast_accel(st, px, G, soft, back=True):
    """Acceleration of asteroids at px (dim, n) from visible massive bodies
    (nbody_kernel.py:166-187 / :343-362); returns (acc, back-reaction)."""
    d = st.dim
    n = px.shape[1]
    acc = np.zeros((d, n))
    bk = np.zeros((d, len(st.mm)))
    for k in range(len(st.mm)):
        if not st.mvis[k]:
            continue
        dx = [st.mx[c, k] - px[c] for c in range(d)]
        f = _pair_force(dx, soft, G)
        f = np.where(st.avis, f, 0.0)
        for c in range(d):
            acc[c] += f * st.mm[k] * dx[c]
            if back:
                bk[c, k] = np.sum((-f) * st.am * dx[c])
    return acc, bk


def _mas_accel(st, bk, G, soft):
    """Massive accelerations: back-reaction + visible massive pairs
    (nbody_kernel.py:196-214 / :377-399)."""
    d, M = st.dim, len(st.mm)
    acc = bk.copy()
    for i in range(M):
        if not st.mvis[i]:
            continue
        for j in range(M):
            if j == i or not st.mvis[j]:
                continue
            dx = [st.mx[c, j] - st.mx[c, i] for c in range(d)]
            f = _pair_force(dx, soft, G)
            for c in range(d):
                acc[c, i] += f * st.mm[j] * dx[c]
    return acc


def frame_launch(st: FrameState, dt_raster, K, m_sub=8, G=G_AU, soft=SOFTENING,
                 max_sub_dt=MAX_SUB_DT_YEARS, max_sub_steps=MAX_SUB_STEPS_PER_FRAME,
                 w1=YOSHIDA_W1, w0=YOSHIDA_W0):
    """One launch of K raster samples; mutates st. Returns dict with
    snap (K, 2d, nAst), snapM (K, 2d, M), subPos (K, m_sub, d, nAst),
    subN (K, nAst), hitT (nAst,) f64 (< 0: none), hitM (nAst,), guard."""
    d, n, M = st.dim, st.ax.shape[1], len(st.mm)
    wd = (w1, w0, w1)
    hitT = np.full(n, -1.0)
    hitM = np.zeros(n, np.int64)
    snap = np.zeros((K, 2 * d, n))
    snapM = np.zeros((K, 2 * d, M))
    subPos = np.zeros((K, max(m_sub, 1), d, n))
    subN = np.zeros((K, n), np.int64)
    # initial accelerations (nbody_kernel.py:151-216)
    aacc, bk = _ast_accel(st, st.ax, G, soft)
    macc = _mas_accel(st, bk, G, soft)
    guard = 0
    for ks in range(K):
        remaining = dt_raster
        while True:
            # dtH (:247-275)
            if remaining <= 1e-12 or guard >= max_sub_steps:
                guard += (remaining > 1e-12)
                break
            guard += 1
            dtH = max_sub_dt
            for i in range(M):
                if not st.mvis[i]:
                    continue
                for j in range(i + 1, M):
                    if not st.mvis[j]:
                        continue
                    dist = np.sqrt(sum((st.mx[c, j] - st.mx[c, i]) ** 2 for c in range(d)))
                    dist = max(dist, 1e-12)
                    vrel = np.sqrt(sum((st.mv[c, j] - st.mv[c, i]) ** 2 for c in range(d)))
                    if vrel > 1e-9:
                        tenc = dist / vrel / 20.0
                        if tenc < dtH:
                            dtH = tenc
            if dtH < max_sub_dt / 1000.0:
                dtH = max_sub_dt / 1000.0
            if dtH > remaining:
                dtH = remaining
            remaining -= dtH
            # hot classification (:283-301)
            hot = np.zeros(n, bool)
            for k in range(M):
                if not st.mvis[k]:
                    continue
                dist = np.maximum(np.sqrt(sum((st.mx[c, k] - st.ax[c]) ** 2 for c in range(d))), 1e-12)
                vrel = np.sqrt(sum((st.mv[c, k] - st.av[c]) ** 2 for c in range(d)))
                hot |= (vrel > 1e-9) & (dist / np.where(vrel > 1e-9, vrel, 1.0) / 20.0 < dtH)
            hot &= st.avis
            mx0 = st.mx.copy()
            calm = st.avis & ~hot
            for w in wd:
                dt = w * dtH
                # phase A (:317-331)
                for c in range(d):
                    st.ax[c] = np.where(calm, st.ax[c] + st.av[c] * dt + 0.5 * aacc[c] * dt * dt, st.ax[c])
                for i in range(M):
                    if st.mvis[i]:
                        for c in range(d):
                            st.mx[c, i] += st.mv[c, i] * dt + 0.5 * macc[c, i] * dt * dt
                # phase B (:343-362): all visible asteroids give back-reaction
                anew, bk = _ast_accel(st, st.ax, G, soft)
                for c in range(d):
                    st.av[c] = np.where(calm, st.av[c] + 0.5 * (aacc[c] + anew[c]) * dt, st.av[c])
                    aacc[c] = np.where(calm, anew[c], aacc[c])
                # phase C (:377-399)
                mnew = _mas_accel(st, bk, G, soft)
                for i in range(M):
                    if st.mvis[i]:
                        for c in range(d):
                            st.mv[c, i] += 0.5 * (macc[c, i] + mnew[c, i]) * dt
                macc = mnew
            # private fine loop of hot asteroids (:416-535)
            tSeg0 = dt_raster - remaining - dtH
            subDt = dt_raster / m_sub if m_sub > 0 else 0.0
            for i in np.flatnonzero(hot):
                p = st.ax[:, i].copy()
                v = st.av[:, i].copy()
                sgn = 1.0 if dtH >= 0.0 else -1.0
                span = abs(dtH)
                tau = 0.0
                guardF = 0
                while tau < span - 1e-15 and guardF < 8000:
                    guardF += 1
                    al = tau / span
                    dtF = max_sub_dt
                    for k in range(M):
                        if not st.mvis[k]:
                            continue
                        mi = [mx0[c, k] + (st.mx[c, k] - mx0[c, k]) * al for c in range(d)]
                        dist = max(np.sqrt(sum((mi[c] - p[c]) ** 2 for c in range(d))), 1e-12)
                        if hitT[i] < 0.0 and dist <= st.mrad[k] + st.arad[i]:
                            hitT[i] = np.float32(ks * dt_raster + tSeg0 + tau)
                            hitM[i] = k
                        vrel = np.sqrt(sum((st.mv[c, k] - v[c]) ** 2 for c in range(d)))
                        if vrel > 1e-9:
                            te = dist / vrel / 20.0
                            if te < dtF:
                                dtF = te
                    if dtF < max_sub_dt / 1000.0:
                        dtF = max_sub_dt / 1000.0
                    if dtF > span - tau:
                        dtF = span - tau
                    if m_sub > 0:
                        tAbs = tSeg0 + tau
                        jn = int(np.floor(tAbs / subDt + 1e-9)) + 1
                        if jn <= m_sub:
                            rest = jn * subDt - tAbs
                            if rest > 0.0 and dtF > rest:
                                dtF = rest
                    tSub = tau
                    for wf in range(3):
                        df = wd[wf] * dtF * sgn
                        a0 = tSub / span
                        acc = _interp_accel(st, mx0, a0, p, G, soft)
                        for c in range(d):
                            p[c] += v[c] * df + 0.5 * acc[c] * df * df
                        tSub += wd[wf] * dtF
                        a1 = tSub / span
                        nacc = _interp_accel(st, mx0, a1, p, G, soft)
                        for c in range(d):
                            v[c] += 0.5 * (acc[c] + nacc[c]) * df
                    tau += dtF
                    if m_sub > 0:
                        q = (tSeg0 + tau) / subDt
                        j = int(np.floor(q + 0.5))
                        if 1 <= j <= m_sub and abs(q - j) < 1e-6:
                            subPos[ks, j - 1, :, i] = p
                            subN[ks, i] += 1
                st.ax[:, i] = p
                st.av[:, i] = v
                acc = _interp_accel(st, mx0, 1.0, p, G, soft, exact_end=True)
                aacc[:, i] = acc
        for c in range(d):
            snap[ks, c] = st.ax[c]
            snap[ks, d + c] = st.av[c]
            snapM[ks, c] = st.mx[c]
            snapM[ks, d + c] = st.mv[c]
    return {"snap": snap, "snapM": snapM, "subPos": subPos, "subN": subN, "hitT": hitT,
            "hitM": hitM, "guard": guard, "aacc": aacc, "macc": macc}


def _interp_accel(st, mx0, al, p, G, soft, exact_end=False):
    d = st.dim
    acc = np.zeros(d)
    for k in range(len(st.mm)):
        if not st.mvis[k]:
            continue
        if exact_end:
            mi = [st.mx[c, k] for c in range(d)]
        else:
            mi = [mx0[c, k] + (st.mx[c, k] - mx0[c, k]) * al for c in range(d)]
        dx = [mi[c] - p[c] for c in range(d)]
        f = _pair_force(dx, soft, G)
        for c in range(d):
            acc[c] += f * st.mm[k] * dx[c]
    return acc


def reference_advance(dt_years, x, y, vx, vy, mass, visible, is_ast, G=G_AU, soft=SOFTENING,
                      max_sub_dt=MAX_SUB_DT_YEARS):
    """Every body on one adaptive Yoshida step (test_kernel.py:16-81)."""
    x, y, vx, vy = (np.array(a, np.float64, copy=True) for a in (x, y, vx, vy))
    vis = np.asarray(visible) != 0
    ast = np.asarray(is_ast) != 0
    mas_i = np.flatnonzero(~ast & vis)

    def accel():
        ax = np.zeros_like(x)
        ay = np.zeros_like(y)
        for i in mas_i:
            dx = x - x[i]
            dy = y - y[i]
            r2 = dx * dx + dy * dy + soft
            f = G / (r2 * np.sqrt(r2))
            f[i] = 0.0
            f[~vis] = 0.0
            sel = vis.copy()
            sel[i] = False
            sel[mas_i[mas_i < i]] = False
            ax[sel] += f[sel] * mass[i] * (-dx[sel])
            ay[sel] += f[sel] * mass[i] * (-dy[sel])
            ax[i] += np.sum(f[sel] * mass[sel] * dx[sel])
            ay[i] += np.sum(f[sel] * mass[sel] * dy[sel])
        return ax, ay

    def adapt_dt():
        dt = max_sub_dt
        for i in mas_i:
            sel = vis.copy()
            sel[i] = False
            sel[mas_i[mas_i < i]] = False
            dist = np.maximum(np.hypot(x[sel] - x[i], y[sel] - y[i]), 1e-12)
            vrel = np.hypot(vx[sel] - vx[i], vy[sel] - vy[i])
            ok = vrel > 1e-9
            if ok.any():
                dt = min(dt, float(np.min(dist[ok] / vrel[ok])) / 20.0)
        return max(dt, max_sub_dt / 1000.0)

    ax, ay = accel()

    def verlet(dt):
        nonlocal ax, ay
        x[vis] += vx[vis] * dt + 0.5 * ax[vis] * dt * dt
        y[vis] += vy[vis] * dt + 0.5 * ay[vis] * dt * dt
        nax, nay = accel()
        vx[vis] += 0.5 * (ax[vis] + nax[vis]) * dt
        vy[vis] += 0.5 * (ay[vis] + nay[vis]) * dt
        ax, ay = nax, nay

    remaining, guard = dt_years, 0
    while remaining > 1e-12 and guard < 100_000:
        guard += 1
        sub = min(remaining, adapt_dt())
        for w in (YOSHIDA_W1, YOSHIDA_W0, YOSHIDA_W1):
            verlet(w * sub)
        remaining -= sub
    return x, y, vx, vy
