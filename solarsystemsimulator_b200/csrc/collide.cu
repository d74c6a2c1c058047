// Collision response of the asteroid films on sm_100a: the merge sweep of
// the massive bodies and the bounce response of asteroid pairs, replacing
// the per-sample host/array code of the reference's film producer
// (analyze_merge, film_producer.py:707-779; bounce_deltas, :916-1019).
//
// Sweep: every alive massive body against every body, the segment of this
// sample (previous -> current position) and the extrapolated segment (current
// -> current + v dt) against the sphere of radius r_m + r_j, in f32 with one
// rounding per operation as the reference's element-wise CuPy code; hits in
// row-major (massive, body) order with the fraction of the raster at the
// closest point; runaways (v^2 > 9 v_esc^2 from the barycentre of the
// massive bodies) in ascending order. The barycentre sums follow NumPy's
// pairwise summation so they carry the reference's rounding.
//
// Bounce: broadphase hits sorted by (offset, a, b) (the reference's order),
// the one-hit-per-body rule applied greedily in that order by one thread
// over a shared-memory bit set, then impulse (restitution e) and overlap
// push per kept hit in f64 on values upcast from the f32 snapshot, each
// operation separately rounded as NumPy evaluates them; the bodies touched
// by an active hit are returned in ascending order with their deltas
// (dx, dy, dvx, dvy).
//
// Both entry points are synchronous (they return counts to the host, as
// sss_broadphase does).

#include "devscan.cuh"

#include <algorithm>

namespace {

using sss_dev::exclusive_scan;
using sss_dev::scan_scratch;

constexpr int SW_NT = 256;

struct SweepIn {
    const float *gx, *gy, *gvx, *gvy, *px, *py, *rr;
    const unsigned char *vis, *is_ast;
    long long n;
    float g_dt;
};

// Alive massive bodies (vis and mass > 0, in the given order), their count
// and the barycentre terms: bx, by (f32 as the reference casts them) and
// the f32 escape coefficient 2 G msum.
struct SweepHead {
    int m_alive;
    int has_mass;
    float bx, by, vesc_coef;
    long long alive[SSS_M_MAX];
};

// term q of the sums over the alive massive bodies: mass (which 0), x * mass
// (1), y * mass (2)
__device__ __forceinline__ double head_term(const SweepIn& in, const double* mass, const SweepHead* h, int q,
                                            int which) {
    const long long i = h->alive[q];
    if (which == 0) return mass[i];
    return __dmul_rn((double)(which == 1 ? in.gx[i] : in.gy[i]), mass[i]);
}

// NumPy's pairwise summation (ndarray.sum over a contiguous f64 vector) of
// the k <= 64 terms: k < 8 sequentially from 0; otherwise eight interleaved
// partial sums combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), then the
// tail (NumPy's blocks hold 128 values, so no further splitting occurs).
// Iterative, no local arrays.
__device__ double np_sum_terms(const SweepIn& in, const double* mass, const SweepHead* h, int k, int which) {
    if (k < 8) {
        double r = 0.0;
        for (int q = 0; q < k; ++q) r = __dadd_rn(r, head_term(in, mass, h, q, which));
        return r;
    }
    double r0 = head_term(in, mass, h, 0, which), r1 = head_term(in, mass, h, 1, which);
    double r2 = head_term(in, mass, h, 2, which), r3 = head_term(in, mass, h, 3, which);
    double r4 = head_term(in, mass, h, 4, which), r5 = head_term(in, mass, h, 5, which);
    double r6 = head_term(in, mass, h, 6, which), r7 = head_term(in, mass, h, 7, which);
    int q = 8;
    for (; q < k - (k % 8); q += 8) {
        r0 = __dadd_rn(r0, head_term(in, mass, h, q, which));
        r1 = __dadd_rn(r1, head_term(in, mass, h, q + 1, which));
        r2 = __dadd_rn(r2, head_term(in, mass, h, q + 2, which));
        r3 = __dadd_rn(r3, head_term(in, mass, h, q + 3, which));
        r4 = __dadd_rn(r4, head_term(in, mass, h, q + 4, which));
        r5 = __dadd_rn(r5, head_term(in, mass, h, q + 5, which));
        r6 = __dadd_rn(r6, head_term(in, mass, h, q + 6, which));
        r7 = __dadd_rn(r7, head_term(in, mass, h, q + 7, which));
    }
    double res = __dadd_rn(__dadd_rn(__dadd_rn(r0, r1), __dadd_rn(r2, r3)),
                           __dadd_rn(__dadd_rn(r4, r5), __dadd_rn(r6, r7)));
    for (; q < k; ++q) res = __dadd_rn(res, head_term(in, mass, h, q, which));
    return res;
}

__global__ void k_sweep_head(const SweepIn in, const double* __restrict__ mass, const long long* __restrict__ m_idx,
                             int m_count, double G, SweepHead* head) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int k = 0;
    for (int q = 0; q < m_count && q < SSS_M_MAX; ++q) {
        const long long i = m_idx[q];
        if (i < 0 || i >= in.n) continue;
        if (in.vis[i] != 0 && mass[i] > 0.0) head->alive[k++] = i;
    }
    head->m_alive = k;
    head->has_mass = 0;
    if (k == 0) return;
    const double msum = np_sum_terms(in, mass, head, k, 0);
    if (msum > 0.0) {
        head->has_mass = 1;
        head->bx = (float)__ddiv_rn(np_sum_terms(in, mass, head, k, 1), msum);
        head->by = (float)__ddiv_rn(np_sum_terms(in, mass, head, k, 2), msum);
        head->vesc_coef = (float)__dmul_rn(__dmul_rn(2.0, G), msum);
    }
}

// f32 segment p0 -> p1 against the sphere (cx, cy, rsum2); returns hit, tt
__device__ __forceinline__ bool seg_hit(float p0x, float p0y, float p1x, float p1y, float cx, float cy,
                                        float rsum2, float& tt) {
    const float ssx = __fsub_rn(p1x, p0x), ssy = __fsub_rn(p1y, p0y);
    const float seg2 = __fadd_rn(__fmul_rn(ssx, ssx), __fmul_rn(ssy, ssy));
    const float den = seg2 > 0.0f ? seg2 : 1.0f;
    float t = __fdiv_rn(__fadd_rn(__fmul_rn(__fsub_rn(cx, p0x), ssx), __fmul_rn(__fsub_rn(cy, p0y), ssy)), den);
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    const float ddx = __fsub_rn(__fadd_rn(p0x, __fmul_rn(t, ssx)), cx);
    const float ddy = __fsub_rn(__fadd_rn(p0y, __fmul_rn(t, ssy)), cy);
    tt = t;
    return __fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)) <= rsum2;
}

__device__ __forceinline__ bool sweep_pair(const SweepIn& in, const SweepHead& h, int row, long long j, float& frac) {
    const long long m = h.alive[row];
    if (j == m || in.vis[j] == 0) return false;
    const float cx = in.gx[m], cy = in.gy[m];
    const float rsum = __fadd_rn(in.rr[m], in.rr[j]);
    const float rsum2 = __fmul_rn(rsum, rsum);
    const float gx = in.gx[j], gy = in.gy[j];
    float ta, tb;
    const bool ha = seg_hit(in.px[j], in.py[j], gx, gy, cx, cy, rsum2, ta);
    const float ex = __fadd_rn(gx, __fmul_rn(in.gvx[j], in.g_dt));
    const float ey = __fadd_rn(gy, __fmul_rn(in.gvy[j], in.g_dt));
    const bool hb = seg_hit(gx, gy, ex, ey, cx, cy, rsum2, tb);
    frac = ha ? __fsub_rn(ta, 1.0f) : tb;
    return ha || hb;
}

__global__ void __launch_bounds__(SW_NT) k_sweep_flags(const SweepIn in, const SweepHead* __restrict__ head,
                                                       int rows, long long* __restrict__ flags) {
    const long long t = (long long)blockIdx.x * SW_NT + threadIdx.x;
    if (t >= (long long)rows * in.n) return;
    const int row = (int)(t / in.n);
    const long long j = t % in.n;
    float frac;
    flags[t] = (row < head->m_alive && sweep_pair(in, *head, row, j, frac)) ? 1 : 0;
}

__global__ void __launch_bounds__(SW_NT) k_sweep_write(const SweepIn in, const SweepHead* __restrict__ head, int rows,
                                                       const long long* __restrict__ flags,
                                                       const long long* __restrict__ pos, int* __restrict__ out,
                                                       long long cap) {
    const long long t = (long long)blockIdx.x * SW_NT + threadIdx.x;
    if (t >= (long long)rows * in.n || !flags[t]) return;
    const int row = (int)(t / in.n);
    const long long j = t % in.n;
    float frac;
    sweep_pair(in, *head, row, j, frac);
    const long long q = pos[t];
    if (q >= cap) return;
    out[3 * q] = (int)head->alive[row];
    out[3 * q + 1] = (int)j;
    out[3 * q + 2] = __float_as_int(frac);
}

__device__ __forceinline__ bool runaway(const SweepIn& in, const SweepHead& h, long long j) {
    if (!h.has_mass || in.vis[j] == 0 || in.is_ast[j] == 0) return false;
    const float dx = __fsub_rn(in.gx[j], h.bx), dy = __fsub_rn(in.gy[j], h.by);
    const float r = fmaxf(sss_hypot_f32(dx, dy), 1e-6f);
    const float v2 = __fadd_rn(__fmul_rn(in.gvx[j], in.gvx[j]), __fmul_rn(in.gvy[j], in.gvy[j]));
    const float vesc2 = __fdiv_rn(h.vesc_coef, r);
    return v2 > __fmul_rn(9.0f, vesc2);
}

__global__ void __launch_bounds__(SW_NT) k_run_flags(const SweepIn in, const SweepHead* __restrict__ head,
                                                     long long* __restrict__ flags) {
    const long long j = (long long)blockIdx.x * SW_NT + threadIdx.x;
    if (j >= in.n) return;
    flags[j] = (head->m_alive > 0 && runaway(in, *head, j)) ? 1 : 0;
}

__global__ void __launch_bounds__(SW_NT) k_run_write(long long n, const long long* __restrict__ flags,
                                                     const long long* __restrict__ pos, int* __restrict__ out,
                                                     long long cap) {
    const long long j = (long long)blockIdx.x * SW_NT + threadIdx.x;
    if (j >= n || !flags[j]) return;
    const long long q = pos[j];
    if (q < cap) out[q] = (int)j;
}

// ------------------------------------------------------------- bounce

constexpr int BF_NT = 256;

__global__ void k_hit_keys(const int* __restrict__ hits, long long n_hits, unsigned long long* __restrict__ keys,
                           unsigned* __restrict__ vals) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_hits) return;
    keys[i] = ((unsigned long long)(unsigned)hits[3 * i] << 42) | ((unsigned long long)(unsigned)hits[3 * i + 1] << 21) |
              (unsigned long long)(unsigned)hits[3 * i + 2];
    vals[i] = (unsigned)i;
}

// The one-hit-per-body rule (bounce_deltas: in (offset, a, b) order a hit
// is kept when neither body is in a hit kept before it) is the
// lexicographically first maximal matching of the hit graph, computed here
// in rounds by one block: an undecided hit whose index is the smallest among
// the undecided hits of both its bodies is kept; then every undecided hit
// touching a body of a kept hit is dropped. Each kept hit is kept by the
// sequential rule too (every earlier hit at its bodies was dropped, and a
// hit is only ever dropped by a kept hit of smaller index, which keeps
// before it), and each round keeps at least the smallest undecided hit.
// After MATCH_ROUNDS rounds, whatever is still undecided is finished by the
// sequential rule in order.
constexpr int MATCH_NT = 1024;
constexpr int MATCH_ROUNDS = 64;

__device__ __forceinline__ void hit_bodies(unsigned long long key, unsigned& a, unsigned& b) {
    a = (unsigned)((key >> 21) & 0x1FFFFFull);
    b = (unsigned)(key & 0x1FFFFFull);
}

__global__ void __launch_bounds__(MATCH_NT) k_bounce_filter(const unsigned long long* __restrict__ keys,
                                                            long long n_hits, int* __restrict__ min_hit,
                                                            unsigned char* __restrict__ taken,
                                                            unsigned char* __restrict__ state,
                                                            long long* __restrict__ keep) {
    __shared__ int s_left[MATCH_NT / 32];
    for (long long i = threadIdx.x; i < n_hits; i += MATCH_NT) {
        unsigned a, b;
        hit_bodies(keys[i], a, b);
        min_hit[a] = INT_MAX;
        min_hit[b] = INT_MAX;
        taken[a] = 0;
        taken[b] = 0;
        state[i] = 0;                                  // 0 undecided, 1 kept, 2 dropped
    }
    __syncthreads();
    int left = 1;
    for (int round = 0; round < MATCH_ROUNDS && left > 0; ++round) {
        for (long long i = threadIdx.x; i < n_hits; i += MATCH_NT) {
            if (__ldcg(state + i)) continue;
            unsigned a, b;
            hit_bodies(keys[i], a, b);
            atomicMin(min_hit + a, (int)i);
            atomicMin(min_hit + b, (int)i);
        }
        __syncthreads();
        for (long long i = threadIdx.x; i < n_hits; i += MATCH_NT) {
            if (__ldcg(state + i)) continue;
            unsigned a, b;
            hit_bodies(keys[i], a, b);
            if (__ldcg(min_hit + a) == (int)i && __ldcg(min_hit + b) == (int)i) {
                state[i] = 1;
                taken[a] = 1;
                taken[b] = 1;
            }
        }
        __syncthreads();
        int mine = 0;
        for (long long i = threadIdx.x; i < n_hits; i += MATCH_NT) {
            if (__ldcg(state + i)) continue;
            unsigned a, b;
            hit_bodies(keys[i], a, b);
            if (__ldcg(taken + a) | __ldcg(taken + b)) {
                state[i] = 2;
            } else {
                min_hit[a] = INT_MAX;
                min_hit[b] = INT_MAX;
                ++mine;
            }
        }
        mine = __reduce_add_sync(0xffffffffu, mine);
        if ((threadIdx.x & 31) == 0) s_left[threadIdx.x >> 5] = mine;
        __syncthreads();
        left = 0;
        for (int w = 0; w < MATCH_NT / 32; ++w) left += s_left[w];
        __syncthreads();
    }
    if (left > 0 && threadIdx.x == 0) {                // the sequential rule for the rest, in order
        for (long long i = 0; i < n_hits; ++i) {
            if (__ldcg(state + i)) continue;
            unsigned a, b;
            hit_bodies(keys[i], a, b);
            if (__ldcg(taken + a) | __ldcg(taken + b)) {
                state[i] = 2;
            } else {
                state[i] = 1;
                taken[a] = 1;
                taken[b] = 1;
            }
        }
    }
    __syncthreads();
    for (long long i = threadIdx.x; i < n_hits; i += MATCH_NT) keep[i] = __ldcg(state + i) == 1;
}

struct BounceIn {
    const float *x, *y, *vx, *vy;
    const double *rr, *mass;
    long long n;
    double dt_y, e;
};

// Impulse and overlap push of kept hit (a, b); returns whether the hit is
// active (approaching at contact) and writes the deltas of both bodies.
__device__ bool bounce_pair(const BounceIn& in, long long a, long long b, double* da, double* db) {
    const double dpx = __dsub_rn((double)in.x[b], (double)in.x[a]);
    const double dpy = __dsub_rn((double)in.y[b], (double)in.y[a]);
    const double dvx = __dsub_rn((double)in.vx[b], (double)in.vx[a]);
    const double dvy = __dsub_rn((double)in.vy[b], (double)in.vy[a]);
    const double dv2 = __dadd_rn(__dmul_rn(dvx, dvx), __dmul_rn(dvy, dvy));
    const double touch = __dadd_rn(in.rr[a], in.rr[b]);
    const double tt2 = __dmul_rn(touch, touch);
    const double c_ = __dsub_rn(__dadd_rn(__dmul_rn(dpx, dpx), __dmul_rn(dpy, dpy)), tt2);
    const double b_ = __dmul_rn(2.0, __dadd_rn(__dmul_rn(dpx, dvx), __dmul_rn(dpy, dvy)));
    const double disc = __dsub_rn(__dmul_rn(b_, b_), __dmul_rn(__dmul_rn(4.0, dv2), c_));
    const double sq = __dsqrt_rn(fmax(disc, 0.0));
    double t_enter = __ddiv_rn(__dsub_rn(-b_, sq), __dmul_rn(2.0, dv2 > 0.0 ? dv2 : 1.0));
    if (isnan(t_enter)) t_enter = 0.0;
    double t_c = 0.0;
    if (!(c_ < 0.0)) t_c = fmin(fmax(t_enter, -in.dt_y), in.dt_y);
    const bool valid = (c_ < 0.0) || (disc >= __dmul_rn(-tt2, 0.01));
    const double ncx = __dadd_rn(dpx, __dmul_rn(dvx, t_c));
    const double ncy = __dadd_rn(dpy, __dmul_rn(dvy, t_c));
    double dist = hypot(ncx, ncy);
    if (!(dist > 1e-30)) dist = 1.0;
    const double nx = __ddiv_rn(ncx, dist), ny = __ddiv_rn(ncy, dist);
    const double vrel = __dadd_rn(__dmul_rn(dvx, nx), __dmul_rn(dvy, ny));
    if (!(valid && vrel < 0.0)) return false;
    const double mi = in.mass[a], mj = in.mass[b];
    double imp = __ddiv_rn(__dmul_rn(-(1.0 + in.e), vrel), __dadd_rn(__ddiv_rn(1.0, mi), __ddiv_rn(1.0, mj)));
    if (isnan(imp)) imp = 0.0;
    else if (isinf(imp)) imp = imp > 0.0 ? 1.7976931348623157e308 : -1.7976931348623157e308;
    da[0] = 0.0;
    da[1] = 0.0;
    da[2] = __dsub_rn(0.0, __ddiv_rn(__dmul_rn(imp, nx), mi));
    da[3] = __dsub_rn(0.0, __ddiv_rn(__dmul_rn(imp, ny), mi));
    db[0] = 0.0;
    db[1] = 0.0;
    db[2] = __dadd_rn(0.0, __ddiv_rn(__dmul_rn(imp, nx), mj));
    db[3] = __dadd_rn(0.0, __ddiv_rn(__dmul_rn(imp, ny), mj));
    const double pdist = hypot(dpx, dpy);
    const double overlap = __dsub_rn(touch, pdist);
    if (overlap > 0.0 && pdist > 1e-30) {
        const double pnx = __ddiv_rn(dpx, pdist), pny = __ddiv_rn(dpy, pdist);
        const double mges = __dadd_rn(mi, mj);
        const double wa = __ddiv_rn(mj, mges), wb = __ddiv_rn(mi, mges);
        const double shift = __dmul_rn(overlap, 1.1);
        da[0] = __dsub_rn(0.0, __dmul_rn(__dmul_rn(pnx, shift), wa));
        da[1] = __dsub_rn(0.0, __dmul_rn(__dmul_rn(pny, shift), wa));
        db[0] = __dadd_rn(0.0, __dmul_rn(__dmul_rn(pnx, shift), wb));
        db[1] = __dadd_rn(0.0, __dmul_rn(__dmul_rn(pny, shift), wb));
    }
    return true;
}

// per kept hit: active flag, deltas into the dense per-body array, touched marks
__global__ void __launch_bounds__(BF_NT) k_bounce_apply(const BounceIn in, const unsigned long long* __restrict__ keys,
                                                        const long long* __restrict__ keep, long long n_hits,
                                                        long long* __restrict__ act, double* __restrict__ dd,
                                                        long long* __restrict__ touched) {
    const long long i = (long long)blockIdx.x * BF_NT + threadIdx.x;
    if (i >= n_hits) return;
    act[i] = 0;
    if (!keep[i]) return;
    const long long a = (long long)((keys[i] >> 21) & 0x1FFFFFull), b = (long long)(keys[i] & 0x1FFFFFull);
    double da[4], db[4];
    if (!bounce_pair(in, a, b, da, db)) return;
    act[i] = 1;
    // one kept hit per body: no two threads write the same rows
    for (int c = 0; c < 4; ++c) {
        dd[4 * a + c] = da[c];
        dd[4 * b + c] = db[c];
    }
    touched[a] = 1;
    touched[b] = 1;
}

__global__ void k_bounce_pairs_out(const unsigned long long* __restrict__ keys, const long long* __restrict__ act,
                                   const long long* __restrict__ pos, long long n_hits, int* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_hits || !act[i]) return;
    const long long q = pos[i];
    out[2 * q] = (int)((keys[i] >> 21) & 0x1FFFFFull);
    out[2 * q + 1] = (int)(keys[i] & 0x1FFFFFull);
}

__global__ void k_bounce_touched_out(long long n, const long long* __restrict__ touched,
                                     const long long* __restrict__ pos, const double* __restrict__ dd,
                                     long long* __restrict__ idx_out, double* __restrict__ d_out) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || !touched[j]) return;
    const long long q = pos[j];
    idx_out[q] = j;
    for (int c = 0; c < 4; ++c) d_out[4 * q + c] = dd[4 * j + c];
}

unsigned nblk(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

size_t al(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

extern "C" int sss_collide_sweep(sss_ctx* ctx, int64_t n, const float* gx, const float* gy, const float* gvx,
                                 const float* gvy, const float* px, const float* py, const float* rr,
                                 const unsigned char* vis, const unsigned char* is_ast, const double* mass,
                                 const int64_t* m_idx, int m_count, double dt_y, double G, int* pairs,
                                 int64_t cap_pairs, int* runaways, int64_t cap_run, int64_t* n_pairs,
                                 int64_t* n_run, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (n < 0 || m_count < 0 || m_count > SSS_M_MAX)
        return sss_set_err(ctx, SSS_ERR_ARG, "bad sizes (n >= 0, 0 <= m_count <= %d)", SSS_M_MAX);
    if (n >= (1LL << 31)) return sss_set_err(ctx, SSS_ERR_ARG, "too many bodies");
    if (!n_pairs || !n_run) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count pointer");
    *n_pairs = 0;
    *n_run = 0;
    if (n == 0 || m_count == 0) return SSS_OK;
    if (!gx || !gy || !gvx || !gvy || !px || !py || !rr || !vis || !is_ast || !mass || !m_idx)
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL input array");
    cudaStream_t st = (cudaStream_t)stream;
    const long long cells = (long long)m_count * n;
    size_t off = 0;
    const size_t o_head = off; off += al(sizeof(SweepHead));
    const size_t o_flags = off; off += al((size_t)cells * 8);
    const size_t o_pos = off; off += al((size_t)cells * 8);
    const size_t o_scan = off; off += al(scan_scratch(cells) * 8);
    const size_t o_rflags = off; off += al((size_t)n * 8);
    const size_t o_rpos = off; off += al((size_t)n * 8);
    const size_t o_rscan = off; off += al(scan_scratch(n) * 8);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* b = (char*)scr;
    SweepHead* head = (SweepHead*)(b + o_head);
    long long* flags = (long long*)(b + o_flags);
    long long* pos = (long long*)(b + o_pos);
    long long* scan = (long long*)(b + o_scan);
    long long* rflags = (long long*)(b + o_rflags);
    long long* rpos = (long long*)(b + o_rpos);
    long long* rscan = (long long*)(b + o_rscan);
    SweepIn in{gx, gy, gvx, gvy, px, py, rr, vis, is_ast, (long long)n, (float)dt_y};
    k_sweep_head<<<1, 32, 0, st>>>(in, mass, (const long long*)m_idx, m_count, G, head);
    SSS_LAUNCH_CHECK(ctx, "k_sweep_head");
    k_sweep_flags<<<nblk(cells, SW_NT), SW_NT, 0, st>>>(in, head, m_count, flags);
    SSS_LAUNCH_CHECK(ctx, "k_sweep_flags");
    SSS_CUDA_TRY(ctx, exclusive_scan(flags, pos, cells, scan, st, ctx->d_status));
    k_run_flags<<<nblk(n, SW_NT), SW_NT, 0, st>>>(in, head, rflags);
    SSS_LAUNCH_CHECK(ctx, "k_run_flags");
    SSS_CUDA_TRY(ctx, exclusive_scan(rflags, rpos, n, rscan, st, ctx->d_status));
    long long tot[2];
    const long long tiles = (cells + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    const long long rtiles = (n + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[0], scan + tiles, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[1], rscan + rtiles, 8, cudaMemcpyDeviceToHost, st));
    // writes stop at the capacities; the totals tell the caller what was found
    k_sweep_write<<<nblk(cells, SW_NT), SW_NT, 0, st>>>(in, head, m_count, flags, pos, pairs, cap_pairs);
    SSS_LAUNCH_CHECK(ctx, "k_sweep_write");
    k_run_write<<<nblk(n, SW_NT), SW_NT, 0, st>>>(n, rflags, rpos, runaways, cap_run);
    SSS_LAUNCH_CHECK(ctx, "k_run_write");
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    *n_pairs = tot[0];
    *n_run = tot[1];
    if (tot[0] > cap_pairs || tot[1] > cap_run)
        return sss_set_err(ctx, SSS_ERR_CAPACITY, "sweep found %lld pairs / %lld runaways (capacity %lld / %lld)",
                           tot[0], tot[1], (long long)cap_pairs, (long long)cap_run);
    return SSS_OK;
}

extern "C" int sss_collide_bounce(sss_ctx* ctx, int64_t n, const float* x, const float* y, const float* vx,
                                  const float* vy, const double* real_r, const double* mass, const int* hits,
                                  int64_t n_hits, double dt_y, double e, int* pairs_out, int64_t* touched_out,
                                  double* deltas_out, int64_t* n_act, int64_t* n_touched, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!n_act || !n_touched) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count pointer");
    *n_act = 0;
    *n_touched = 0;
    if (n < 0 || n_hits < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    // body indices are packed in 21 bits of the sort key
    if (n > SSS_COLLIDE_MAX_BODIES)
        return sss_set_err(ctx, SSS_ERR_ARG, "bounce: at most %d bodies", SSS_COLLIDE_MAX_BODIES);
    if (n_hits == 0 || n == 0) return SSS_OK;
    if (!x || !y || !vx || !vy || !real_r || !mass || !hits || !pairs_out || !touched_out || !deltas_out)
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");

    cudaStream_t st = (cudaStream_t)stream;
    size_t off = 0;
    const size_t o_k0 = off; off += al((size_t)n_hits * 8);
    const size_t o_k1 = off; off += al((size_t)n_hits * 8);
    const size_t o_v0 = off; off += al((size_t)n_hits * 4);
    const size_t o_v1 = off; off += al((size_t)n_hits * 4);
    const size_t o_rs = off; off += al(sss_dev::radix_scratch(n_hits) * 8);
    const size_t o_keep = off; off += al((size_t)n_hits * 8);
    const size_t o_act = off; off += al((size_t)n_hits * 8);
    const size_t o_apos = off; off += al((size_t)n_hits * 8);
    const size_t o_ascan = off; off += al(scan_scratch(n_hits) * 8);
    const size_t o_dd = off; off += al((size_t)n * 32);
    const size_t o_tch = off; off += al((size_t)n * 8);
    const size_t o_tpos = off; off += al((size_t)n * 8);
    const size_t o_tscan = off; off += al(scan_scratch(n) * 8);
    const size_t o_minh = off; off += al((size_t)n * 4);
    const size_t o_taken = off; off += al((size_t)n);
    const size_t o_state = off; off += al((size_t)n_hits);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* b = (char*)scr;
    unsigned long long* k0 = (unsigned long long*)(b + o_k0);
    unsigned long long* k1 = (unsigned long long*)(b + o_k1);
    unsigned* v0 = (unsigned*)(b + o_v0);
    unsigned* v1 = (unsigned*)(b + o_v1);
    long long* keep = (long long*)(b + o_keep);
    long long* act = (long long*)(b + o_act);
    long long* apos = (long long*)(b + o_apos);
    long long* ascan = (long long*)(b + o_ascan);
    double* dd = (double*)(b + o_dd);
    long long* tch = (long long*)(b + o_tch);
    long long* tpos = (long long*)(b + o_tpos);
    long long* tscan = (long long*)(b + o_tscan);
    k_hit_keys<<<nblk(n_hits, 256), 256, 0, st>>>(hits, n_hits, k0, v0);
    SSS_LAUNCH_CHECK(ctx, "k_hit_keys");
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(k0, v0, k1, v1, n_hits, (long long*)(b + o_rs), st, ctx->d_status));
    k_bounce_filter<<<1, MATCH_NT, 0, st>>>(k0, n_hits, (int*)(b + o_minh), (unsigned char*)(b + o_taken),
                                            (unsigned char*)(b + o_state), keep);
    SSS_LAUNCH_CHECK(ctx, "k_bounce_filter");
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(dd, 0, (size_t)n * 32, st));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(tch, 0, (size_t)n * 8, st));
    BounceIn in{x, y, vx, vy, real_r, mass, (long long)n, dt_y, e};
    k_bounce_apply<<<nblk(n_hits, BF_NT), BF_NT, 0, st>>>(in, k0, keep, n_hits, act, dd, tch);
    SSS_LAUNCH_CHECK(ctx, "k_bounce_apply");
    SSS_CUDA_TRY(ctx, exclusive_scan(act, apos, n_hits, ascan, st, ctx->d_status));
    SSS_CUDA_TRY(ctx, exclusive_scan(tch, tpos, n, tscan, st, ctx->d_status));
    k_bounce_pairs_out<<<nblk(n_hits, 256), 256, 0, st>>>(k0, act, apos, n_hits, pairs_out);
    SSS_LAUNCH_CHECK(ctx, "k_bounce_pairs_out");
    k_bounce_touched_out<<<nblk(n, 256), 256, 0, st>>>(n, tch, tpos, dd, (long long*)touched_out, deltas_out);
    SSS_LAUNCH_CHECK(ctx, "k_bounce_touched_out");
    long long tot[2];
    const long long at = (n_hits + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    const long long tt = (n + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[0], ascan + at, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&tot[1], tscan + tt, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    *n_act = tot[0];
    *n_touched = tot[1];
    return SSS_OK;
}

// ------------------------------------------------------------ fragmentation
//
// Asteroid x asteroid impacts far above the pair's escape speed break both
// bodies into n_frag fragments (the asteroid-cloud configuration: above 5 x
// v_esc). The reference's producer only detects a shatter (body x body at
// 1.5 v_esc, film_producer.py:801-822) and leaves the fragments to its
// client's shatter() (index.html:7705-7745): equal fragments on a ring of
// radius r_a + r_b about the centre of mass, scattered velocities with their
// mean removed so that mass and momentum are conserved. Here the same
// construction runs on the device for every active bounce pair whose impact
// speed |v_b - v_a| >= factor * sqrt(2 G (m_a + m_b) / (r_a + r_b)), with the
// client's random numbers replaced by a counter-based generator (SplitMix64
// of the seed, the two body indices and the fragment number), so a film is
// reproducible. Radii keep the volume: r_f = cbrt((r_a^3 + r_b^3) / n_frag).

namespace {

constexpr int FRAG_NT = 128;

__device__ __forceinline__ double frag_uniform(unsigned long long seed, long long a, long long b, int k, int j) {
    unsigned long long h = seed ^ ((unsigned long long)a * 0x9E3779B97F4A7C15ull) ^
                           ((unsigned long long)b * 0xC2B2AE3D27D4EB4Full);
    h += (unsigned long long)(2 * k + j + 1) * 0xD6E8FEB86659FD93ull;
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 31;
    return (double)(h >> 11) * 0x1.0p-53;
}

struct FragIn {
    const float *x, *y, *vx, *vy;
    const double *rr, *mass;
    double G, factor;
    unsigned long long seed;
    int n_frag;
};

__device__ __forceinline__ bool frag_test(const FragIn& in, long long a, long long b) {
    const double ma = in.mass[a], mb = in.mass[b];
    const double mt = ma + mb;
    if (!(mt > 0.0) || !(in.factor > 0.0)) return false;
    const double dvx = (double)in.vx[b] - (double)in.vx[a];
    const double dvy = (double)in.vy[b] - (double)in.vy[a];
    const double v_imp = sqrt(dvx * dvx + dvy * dvy);
    double touch = in.rr[a] + in.rr[b];
    if (touch < 1e-12) touch = 1e-12;
    const double v_esc = sqrt(2.0 * in.G * mt / touch);
    return v_imp >= in.factor * v_esc;
}

__global__ void __launch_bounds__(FRAG_NT) k_frag_flags(const FragIn in, const int* __restrict__ pairs, long long np_,
                                                        long long* __restrict__ flags) {
    const long long t = (long long)blockIdx.x * FRAG_NT + threadIdx.x;
    if (t >= np_) return;
    flags[t] = frag_test(in, pairs[2 * t], pairs[2 * t + 1]) ? 1 : 0;
}

// One thread per fragmenting pair: its n_frag fragments (x, y, vx, vy, m, r).
__global__ void __launch_bounds__(FRAG_NT) k_frag_write(const FragIn in, const int* __restrict__ pairs, long long np_,
                                                        const long long* __restrict__ flags,
                                                        const long long* __restrict__ pos, long long cap,
                                                        int* __restrict__ parents, double* __restrict__ frags) {
    const long long t = (long long)blockIdx.x * FRAG_NT + threadIdx.x;
    if (t >= np_ || !flags[t]) return;
    const long long q = pos[t];
    if (q >= cap) return;
    const long long a = pairs[2 * t], b = pairs[2 * t + 1];
    parents[2 * q] = (int)a;
    parents[2 * q + 1] = (int)b;
    const double ma = in.mass[a], mb = in.mass[b], mt = ma + mb;
    const double xa = in.x[a], ya = in.y[a], xb = in.x[b], yb = in.y[b];
    const double vxa = in.vx[a], vya = in.vy[a], vxb = in.vx[b], vyb = in.vy[b];
    const double cx = (ma * xa + mb * xb) / mt, cy = (ma * ya + mb * yb) / mt;
    const double cvx = (ma * vxa + mb * vxb) / mt, cvy = (ma * vya + mb * vyb) / mt;
    const double dvx = vxb - vxa, dvy = vyb - vya;
    const double v_imp = sqrt(dvx * dvx + dvy * dvy);
    const int N = in.n_frag;
    const double ring = in.rr[a] + in.rr[b];
    const double rf = cbrt((in.rr[a] * in.rr[a] * in.rr[a] + in.rr[b] * in.rr[b] * in.rr[b]) / N);
    const double mf = mt / N;
    double mx = 0.0, my = 0.0;
    for (int k = 0; k < N; ++k) {
        const double ang = 2.0 * M_PI * k / N + (frag_uniform(in.seed, a, b, k, 0) - 0.5) * 0.6;
        const double spd = v_imp * (0.25 + 0.35 * frag_uniform(in.seed, a, b, k, 1));
        mx += cos(ang) * spd;
        my += sin(ang) * spd;
    }
    mx /= N;
    my /= N;
    double* f = frags + q * (long long)N * 6;
    for (int k = 0; k < N; ++k) {
        const double ang = 2.0 * M_PI * k / N + (frag_uniform(in.seed, a, b, k, 0) - 0.5) * 0.6;
        const double spd = v_imp * (0.25 + 0.35 * frag_uniform(in.seed, a, b, k, 1));
        const double th = 2.0 * M_PI * k / N;
        f[6 * k + 0] = cx + cos(th) * ring;
        f[6 * k + 1] = cy + sin(th) * ring;
        f[6 * k + 2] = cvx + (cos(ang) * spd - mx);
        f[6 * k + 3] = cvy + (sin(ang) * spd - my);
        f[6 * k + 4] = mf;
        f[6 * k + 5] = rf;
    }
}

}  // namespace

extern "C" int sss_collide_fragment(sss_ctx* ctx, int64_t n, const float* x, const float* y, const float* vx,
                                    const float* vy, const double* real_r, const double* mass, const int* pairs,
                                    int64_t n_pairs, double G, double factor, int n_frag, uint64_t seed,
                                    int* parents_out, double* frags_out, int64_t cap, int64_t* n_events,
                                    void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!n_events) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count pointer");
    *n_events = 0;
    if (n < 0 || n_pairs < 0 || cap < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n_frag < 2 || n_frag > 16) return sss_set_err(ctx, SSS_ERR_ARG, "n_frag must be in [2, 16]");
    if (!(factor >= 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "factor must be >= 0");
    if (n_pairs == 0 || factor == 0.0) return SSS_OK;
    if (!x || !y || !vx || !vy || !real_r || !mass || !pairs || (cap > 0 && (!parents_out || !frags_out)))
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    cudaStream_t st = (cudaStream_t)stream;
    size_t off = 0;
    const size_t o_flags = off; off += al((size_t)n_pairs * 8);
    const size_t o_pos = off; off += al((size_t)n_pairs * 8);
    const size_t o_scan = off; off += al(scan_scratch(n_pairs) * 8);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* b = (char*)scr;
    long long* flags = (long long*)(b + o_flags);
    long long* pos = (long long*)(b + o_pos);
    long long* scan = (long long*)(b + o_scan);
    FragIn in{x, y, vx, vy, real_r, mass, G, factor, (unsigned long long)seed, n_frag};
    k_frag_flags<<<nblk(n_pairs, FRAG_NT), FRAG_NT, 0, st>>>(in, pairs, n_pairs, flags);
    SSS_LAUNCH_CHECK(ctx, "k_frag_flags");
    SSS_CUDA_TRY(ctx, exclusive_scan(flags, pos, n_pairs, scan, st, ctx->d_status));
    k_frag_write<<<nblk(n_pairs, FRAG_NT), FRAG_NT, 0, st>>>(in, pairs, n_pairs, flags, pos, cap, parents_out,
                                                             frags_out);
    SSS_LAUNCH_CHECK(ctx, "k_frag_write");
    long long tot = 0;
    const long long tiles = (n_pairs + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&tot, scan + tiles, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    *n_events = tot;
    if (tot > cap) return sss_set_err(ctx, SSS_ERR_CAPACITY, "fragment: %lld events, capacity %lld", tot,
                                      (long long)cap);
    return SSS_OK;
}
