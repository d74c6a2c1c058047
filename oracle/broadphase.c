/*
 * CPU oracle — TEST INFRASTRUCTURE ONLY (never linked into libsss or the
 * product path). Plain-C restatement of the broadphase of the reference's
 * film producer, `Erkennungskarte._hits` with `_zellschluessel`
 * (backend/film_producer.py:223-321), for scenes too large for the NumPy
 * restatement (oracle/broadphase.py) to check in seconds:
 *
 *   alive    is_ast && vis && x >= lo && x < hi + (float)halo      (f32, :232-234)
 *   cell     floor((double)x / h), floor((double)y / h) as int64   (:238-239)
 *   key      cx * 73856093 ^ cy * 19349663, int64 wrap-around      (:320-321)
 *   order    stable sort of the alive bodies by key                 (:241-242)
 *   partners for each offset of (0,0) (1,0) (0,1) (1,1) (1,-1), the
 *            bodies whose key equals the offset cell's key (binary
 *            search, :270-273); keep a < b on (0,0), a != b elsewhere
 *            (:285); candidates counted before the keep rule (:274)
 *   f32 test closest approach over t in [-dt, dt] with every operation
 *            rounded to f32 (NumPy's element-wise evaluation, :243-259):
 *            dv2 = dvx dvx + dvy dvy; t = clip(-(dpx dvx + dpy dvy) /
 *            (dv2 > 0 ? dv2 : 1), -dt, dt); hit if (dpx + dvx t)^2 +
 *            (dpy + dvy t)^2 <= (r_a + r_b + 1e-6)^2
 *   owner    min(x_a, x_b) < hi (f32, :296)
 *   f64 test the same closest approach in f64 on the upcast values with
 *            r_a + r_b (:303-314)
 *
 * Hits come out in the reference's order: by offset, then by alive body a
 * (ascending index), then by the partner's position in the sorted order.
 * Compiled with -ffp-contract=off, so the arithmetic is the IEEE evaluation
 * of that operation order. OpenMP over the alive bodies; the per-body hit
 * lists are concatenated in body order, so the result does not depend on
 * the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int64_t key;
    int64_t pos;     /* position among the alive bodies (tie-break: stable) */
} keyed;

static int cmp_keyed(const void* a, const void* b) {
    const keyed* p = (const keyed*)a;
    const keyed* q = (const keyed*)b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return p->pos < q->pos ? -1 : (p->pos > q->pos);
}

static int64_t cell_key(int64_t cx, int64_t cy) {
    const uint64_t a = (uint64_t)cx * 73856093ull;
    const uint64_t b = (uint64_t)cy * 19349663ull;
    return (int64_t)(a ^ b);
}

/* first index with ks[i] >= k (side="left") / > k (side="right") */
static int64_t lower(const int64_t* ks, int64_t n, int64_t k) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t m = lo + (hi - lo) / 2;
        if (ks[m] < k) lo = m + 1; else hi = m;
    }
    return lo;
}

static int64_t upper(const int64_t* ks, int64_t n, int64_t k) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t m = lo + (hi - lo) / 2;
        if (ks[m] <= k) lo = m + 1; else hi = m;
    }
    return lo;
}

static float clipf(float t, float lo, float hi) {   /* np.clip: NaN stays NaN */
    if (t < lo) t = lo;
    if (t > hi) t = hi;
    return t;
}

static double clipd(double t, double lo, double hi) {
    if (t < lo) t = lo;
    if (t > hi) t = hi;
    return t;
}

static int hit_f32(const float* gx, const float* gy, const float* gvx, const float* gvy, const float* rr,
                   int64_t a, int64_t b, float dt) {
    const float dpx = gx[b] - gx[a], dpy = gy[b] - gy[a];
    const float dvx = gvx[b] - gvx[a], dvy = gvy[b] - gvy[a];
    const float dv2 = dvx * dvx + dvy * dvy;
    const float num = -(dpx * dvx + dpy * dvy);
    const float t = clipf(num / (dv2 > 0.0f ? dv2 : 1.0f), -dt, dt);
    const float cx = dpx + dvx * t, cy = dpy + dvy * t;
    const float rs = rr[a] + rr[b] + 1e-6f;
    return cx * cx + cy * cy <= rs * rs;
}

static int hit_f64(const float* gx, const float* gy, const float* gvx, const float* gvy, const float* rr,
                   int64_t a, int64_t b, double dt) {
    const double dpx = (double)gx[b] - (double)gx[a], dpy = (double)gy[b] - (double)gy[a];
    const double dvx = (double)gvx[b] - (double)gvx[a], dvy = (double)gvy[b] - (double)gvy[a];
    const double dv2 = dvx * dvx + dvy * dvy;
    const double num = -(dpx * dvx + dpy * dvy);
    const double t = clipd(num / (dv2 > 0.0 ? dv2 : 1.0), -dt, dt);
    const double cx = dpx + dvx * t, cy = dpy + dvy * t;
    const double rs = (double)rr[a] + (double)rr[b];
    return cx * cx + cy * cy <= rs * rs;
}

/*
 * Returns the number of hits (written to out_i/out_j up to cap) or -1 on an
 * allocation failure; *n_cand receives the candidate count. lo/hi are the
 * stripe bounds as f32 values (use +-inf for the whole line).
 */
int64_t oracle_broadphase_hits(const float* gx, const float* gy, const float* gvx, const float* gvy,
                               const float* rr, const uint8_t* is_ast, const uint8_t* vis, int64_t n,
                               double dt_y, double h, double halo, float lo, float hi, int64_t* out_i,
                               int64_t* out_j, int64_t cap, int64_t* n_cand, int nthreads) {
    static const int OFF[5][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}, {1, -1}};
    if (nthreads < 1) nthreads = 1;
    *n_cand = 0;
    const float hi_halo = hi + (float)halo;
    int64_t na = 0;
    for (int64_t i = 0; i < n; ++i)
        if ((!is_ast || is_ast[i]) && (!vis || vis[i]) && gx[i] >= lo && gx[i] < hi_halo) ++na;
    if (na < 2) return 0;
    int64_t* ai = (int64_t*)malloc(sizeof(int64_t) * na);
    int64_t* cx = (int64_t*)malloc(sizeof(int64_t) * na);
    int64_t* cy = (int64_t*)malloc(sizeof(int64_t) * na);
    keyed* kv = (keyed*)malloc(sizeof(keyed) * na);
    int64_t* ks = (int64_t*)malloc(sizeof(int64_t) * na);
    int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * (na + 1));
    if (!ai || !cx || !cy || !kv || !ks || !cnt) {
        free(ai); free(cx); free(cy); free(kv); free(ks); free(cnt);
        return -1;
    }
    na = 0;
    for (int64_t i = 0; i < n; ++i)
        if ((!is_ast || is_ast[i]) && (!vis || vis[i]) && gx[i] >= lo && gx[i] < hi_halo) ai[na++] = i;
    for (int64_t r = 0; r < na; ++r) {
        cx[r] = (int64_t)floor((double)gx[ai[r]] / h);
        cy[r] = (int64_t)floor((double)gy[ai[r]] / h);
        kv[r].key = cell_key(cx[r], cy[r]);
        kv[r].pos = r;
    }
    qsort(kv, (size_t)na, sizeof(keyed), cmp_keyed);
    for (int64_t r = 0; r < na; ++r) ks[r] = kv[r].key;
    const float dt32 = (float)dt_y;
    int64_t total = 0, cand = 0;
    int failed = 0;
    for (int o = 0; o < 5 && !failed; ++o) {
        const int ox = OFF[o][0], oy = OFF[o][1];
        /* f32 hits per alive body, kept for the ones that also pass ownership and f64 */
        int64_t** lists = (int64_t**)calloc((size_t)na, sizeof(int64_t*));
        if (!lists) { failed = 1; break; }
        int64_t cand_o = 0;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256) reduction(+ : cand_o)
        for (int64_t r = 0; r < na; ++r) {
            const int64_t k2 = cell_key(cx[r] + ox, cy[r] + oy);
            const int64_t c0 = lower(ks, na, k2), c1 = upper(ks, na, k2);
            cand_o += c1 - c0;
            cnt[r] = 0;
            const int64_t a = ai[r];
            int64_t m = 0, room = 0;
            int64_t* buf = NULL;
            for (int64_t c = c0; c < c1; ++c) {
                const int64_t b = ai[kv[c].pos];
                if ((ox == 0 && oy == 0) ? !(a < b) : (a == b)) continue;
                if (!hit_f32(gx, gy, gvx, gvy, rr, a, b, dt32)) continue;
                if (!(fminf(gx[a], gx[b]) < hi)) continue;
                if (!hit_f64(gx, gy, gvx, gvy, rr, a, b, dt_y)) continue;
                if (m == room) {
                    room = room ? 2 * room : 8;
                    int64_t* nb = (int64_t*)realloc(buf, sizeof(int64_t) * room);
                    if (!nb) { free(buf); buf = NULL; m = -1; break; }
                    buf = nb;
                }
                buf[m++] = b;
            }
            lists[r] = buf;
            cnt[r] = m;
        }
        cand += cand_o;
        for (int64_t r = 0; r < na; ++r) {
            if (cnt[r] < 0) { failed = 1; continue; }
            for (int64_t q = 0; q < cnt[r]; ++q) {
                if (total < cap) {
                    out_i[total] = ai[r];
                    out_j[total] = lists[r][q];
                }
                ++total;
            }
            free(lists[r]);
        }
        free(lists);
    }
    free(ai); free(cx); free(cy); free(kv); free(ks); free(cnt);
    *n_cand = cand;
    return failed ? -1 : total;
}
