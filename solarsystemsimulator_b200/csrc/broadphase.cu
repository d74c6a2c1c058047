// Uniform-grid (spatial-hash) asteroid x asteroid collision broadphase for
// sm_100a: replaces `Erkennungskarte._hits` + `_zellschluessel` (reference
// backend/film_producer.py:223-321).
//
// The colliding-pair list is bit-exact against the reference on the same f32
// snapshot, so every step keeps the reference's arithmetic:
// * alive = asteroid & visible & x >= lo & x < hi + f32(halo)   (f32)
// * cell = floor(f64(x) / h) as int64; key = cx*73856093 ^ cy*19349663 with
//   int64 wrap-around; bodies stably sorted by key; for each of the five
//   neighbour offsets (0,0) (1,0) (0,1) (1,1) (1,-1) the candidates of a body
//   are the bodies whose key equals the offset cell's key (hash collisions
//   included, as in the reference's searchsorted ranges);
// * (0,0) keeps a < b, the other offsets a != b;
// * f32 closest approach over t in [-dt, dt] with every operation rounded
//   separately (the reference evaluates it as separate element-wise array
//   operations, so no fused multiply-add may appear), radii + 1e-6;
// * ownership: min(x_a, x_b) < hi (f32); exact recheck in f64 of the f32
//   values, again without contraction.
// The candidate list is never materialised: one kernel walks the flattened
// candidate index space (offset-major, then body, then range position — the
// reference's expansion order) in contiguous chunks per warp, one candidate
// per lane, tests each pair and appends hits; the partners' values are read
// from records stored in sorted-key order (one gather per call), so the
// lanes of a warp read consecutive records. The host
// sorts the hits by (offset, a, b), which is the reference's output order.

#include "devscan.cuh"

namespace {

constexpr int BP_NT = 256;
constexpr int BP_CHUNK = 8192;   // consecutive candidates per warp

__device__ __forceinline__ long long cell_key(long long cx, long long cy) {
    // int64 wrap-around multiply (the reference's `cx * int64(73856093) ^ cy * int64(19349663)`)
    const unsigned long long a = (unsigned long long)cx * 73856093ull;
    const unsigned long long b = (unsigned long long)cy * 19349663ull;
    return (long long)(a ^ b);
}

__device__ __forceinline__ bool alive_of(const unsigned char* is_ast, const unsigned char* vis, const float* x,
                                         long long i, float lo, float hi_halo) {
    return is_ast[i] && vis[i] != 0 && x[i] >= lo && x[i] < hi_halo;
}

__global__ void __launch_bounds__(BP_NT) k_alive_count(const unsigned char* __restrict__ is_ast,
                                                       const unsigned char* __restrict__ vis,
                                                       const float* __restrict__ x, long long n, float lo,
                                                       float hi_halo, long long* __restrict__ counts) {
    const long long base = (long long)blockIdx.x * sss_dev::SCAN_TILE;
    long long c = 0;
    for (int k = 0; k < sss_dev::SCAN_ITEMS; ++k) {
        const long long i = base + (long long)threadIdx.x * sss_dev::SCAN_ITEMS + k;
        if (i < n && alive_of(is_ast, vis, x, i, lo, hi_halo)) ++c;
    }
    long long tot;
    sss_dev::block_exclusive_scan(c, &tot);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

// Compaction in ascending body order + cell and key of every alive body.
__global__ void __launch_bounds__(BP_NT) k_alive_scatter(const unsigned char* __restrict__ is_ast,
                                                         const unsigned char* __restrict__ vis,
                                                         const float* __restrict__ x, const float* __restrict__ y,
                                                         long long n, float lo, float hi_halo, double h,
                                                         const long long* __restrict__ offs,
                                                         unsigned* __restrict__ ai, long long* __restrict__ cx,
                                                         long long* __restrict__ cy,
                                                         unsigned long long* __restrict__ skey,
                                                         unsigned* __restrict__ sval) {
    const long long base = (long long)blockIdx.x * sss_dev::SCAN_TILE;
    bool f[sss_dev::SCAN_ITEMS];
    long long c = 0;
    for (int k = 0; k < sss_dev::SCAN_ITEMS; ++k) {
        const long long i = base + (long long)threadIdx.x * sss_dev::SCAN_ITEMS + k;
        f[k] = i < n && alive_of(is_ast, vis, x, i, lo, hi_halo);
        c += f[k];
    }
    long long tot;
    long long r = sss_dev::block_exclusive_scan(c, &tot) + offs[blockIdx.x];
    for (int k = 0; k < sss_dev::SCAN_ITEMS; ++k) {
        if (!f[k]) continue;
        const long long i = base + (long long)threadIdx.x * sss_dev::SCAN_ITEMS + k;
        const long long ix = (long long)floor(__ddiv_rn((double)x[i], h));
        const long long iy = (long long)floor(__ddiv_rn((double)y[i], h));
        ai[r] = (unsigned)i;
        cx[r] = ix;
        cy[r] = iy;
        // signed int64 order as unsigned: flip the sign bit
        skey[r] = (unsigned long long)cell_key(ix, iy) ^ 0x8000000000000000ull;
        sval[r] = (unsigned)r;
        ++r;
    }
}

__device__ __forceinline__ long long lower_bound(const unsigned long long* a, long long n, unsigned long long v) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ long long upper_bound(const unsigned long long* a, long long n, unsigned long long v) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid] <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__constant__ int c_off[5][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}, {1, -1}};   // film_producer.py:155

// Key range of every (offset, body) segment: start in the sorted keys and length.
__global__ void k_ranges(const long long* __restrict__ cx, const long long* __restrict__ cy, long long na,
                         const unsigned long long* __restrict__ ks, long long* __restrict__ seg_lo,
                         long long* __restrict__ seg_len) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 5 * na) return;
    const int o = (int)(t / na);
    const long long r = t - (long long)o * na;
    const unsigned long long k2 =
        (unsigned long long)cell_key(cx[r] + c_off[o][0], cy[r] + c_off[o][1]) ^ 0x8000000000000000ull;
    const long long lo = lower_bound(ks, na, k2);
    const long long hi = upper_bound(ks, na, k2);
    seg_lo[t] = lo;
    seg_len[t] = hi - lo;
}

struct Hit {
    int o;
    unsigned a, b;
};

// A body's snapshot values as the tests read them.
struct Body {
    float x, y, vx, vy, rr;
};

// f32 closest-approach prefilter (film_producer.py:241-259), op by op.
__device__ __forceinline__ bool ccd_f32(const Body& A, const Body& B, float dtf) {
    const float dpx = __fsub_rn(B.x, A.x);
    const float dpy = __fsub_rn(B.y, A.y);
    const float dvx = __fsub_rn(B.vx, A.vx);
    const float dvy = __fsub_rn(B.vy, A.vy);
    const float dv2 = __fadd_rn(__fmul_rn(dvx, dvx), __fmul_rn(dvy, dvy));
    const float num = -__fadd_rn(__fmul_rn(dpx, dvx), __fmul_rn(dpy, dvy));
    const float t = fminf(fmaxf(__fdiv_rn(num, dv2 > 0.f ? dv2 : 1.0f), -dtf), dtf);
    const float cxm = __fadd_rn(dpx, __fmul_rn(dvx, t));
    const float cym = __fadd_rn(dpy, __fmul_rn(dvy, t));
    const float rsum = __fadd_rn(__fadd_rn(A.rr, B.rr), 1e-6f);
    return __fadd_rn(__fmul_rn(cxm, cxm), __fmul_rn(cym, cym)) <= __fmul_rn(rsum, rsum);
}

// exact recheck in f64 of the f32 values (film_producer.py:303-314)
__device__ __forceinline__ bool ccd_f64(const Body& A, const Body& B, double dt) {
    const double dpx = __dsub_rn((double)B.x, (double)A.x);
    const double dpy = __dsub_rn((double)B.y, (double)A.y);
    const double dvx = __dsub_rn((double)B.vx, (double)A.vx);
    const double dvy = __dsub_rn((double)B.vy, (double)A.vy);
    const double dv2 = __dadd_rn(__dmul_rn(dvx, dvx), __dmul_rn(dvy, dvy));
    const double num = -__dadd_rn(__dmul_rn(dpx, dvx), __dmul_rn(dpy, dvy));
    const double t = fmin(fmax(__ddiv_rn(num, dv2 > 0.0 ? dv2 : 1.0), -dt), dt);
    const double cxm = __dadd_rn(dpx, __dmul_rn(dvx, t));
    const double cym = __dadd_rn(dpy, __dmul_rn(dvy, t));
    const double rsum = __dadd_rn((double)A.rr, (double)B.rr);
    return __dadd_rn(__dmul_rn(cxm, cxm), __dmul_rn(cym, cym)) <= __dmul_rn(rsum, rsum);
}

// Body records in sorted-key order: position pos holds the body of row
// order[pos] (x, y, vx, vy | rr bits, body index), so a segment's partners
// are read from consecutive records instead of through two index arrays.
__global__ void k_sorted_records(const float* __restrict__ x, const float* __restrict__ y,
                                 const float* __restrict__ vx, const float* __restrict__ vy,
                                 const float* __restrict__ rr, const unsigned* __restrict__ ai,
                                 const unsigned* __restrict__ order, long long na, float4* __restrict__ rec,
                                 uint2* __restrict__ rec2) {
    const long long pos = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= na) return;
    const unsigned b = ai[order[pos]];
    rec[pos] = make_float4(x[b], y[b], vx[b], vy[b]);
    rec2[pos] = make_uint2(__float_as_uint(rr[b]), b);
}

struct CandArgs {
    const float *x, *y, *vx, *vy, *rr;
    const unsigned* ai;          // row -> body
    const float4* rec;           // sorted position -> (x, y, vx, vy) of its body
    const uint2* rec2;           // sorted position -> (rr bits, body)
    const long long* seg_lo;     // [5*na]
    const long long* seg_start;  // [5*na + 1] exclusive prefix of segment lengths
    long long n_seg, total;
    float dtf, hi;
    double dt;
    Hit* hits;
    long long cap;
    unsigned long long* n_hits;
};

__device__ __forceinline__ long long find_segment(const long long* start, long long n_seg, long long idx) {
    // last s with start[s] <= idx
    long long lo = 0, hi = n_seg;
    while (hi - lo > 1) {
        const long long mid = (lo + hi) >> 1;
        if (start[mid] <= idx) lo = mid; else hi = mid;
    }
    return lo;
}

// keep rule, f32 prefilter, ownership, f64 recheck, append (film_producer.py:241-314)
// Pairs that provably fail the f32 test are skipped before it. For every t
// in [-dt, dt], |dp + dv t| >= |dp| - (|dvx| + |dvy|) dt; if |dp| exceeds
// twice reach = (|dvx| + |dvy|) dt + rsum, the closest approach is at least
// 2 rsum. The f32 evaluation of the test errs by a few ulp of |dp|, below
// 1e-7 AU while |dp| < 1 AU, while rsum >= 1e-6 AU (radii + 1e-6), so such
// a pair can never pass it: the skip changes no result, only the work.
__device__ __forceinline__ bool surely_apart(const Body& A, const Body& B, float dtf) {
    const float dpx = B.x - A.x, dpy = B.y - A.y;
    const float dp2 = dpx * dpx + dpy * dpy;
    const float reach = (fabsf(B.vx - A.vx) + fabsf(B.vy - A.vy)) * dtf + (A.rr + B.rr + 1e-6f);
    return dp2 < 1.0f && dp2 > 4.0001f * reach * reach;
}

__device__ __forceinline__ void test_pair(const CandArgs& a, int o, unsigned ab, const Body& A, uint2 q, float4 v) {
    const unsigned bb = q.y;
    const bool keep = (o == 0) ? (ab < bb) : (ab != bb);
    if (!keep) return;
    const Body B{v.x, v.y, v.z, v.w, __uint_as_float(q.x)};
    if (surely_apart(A, B, a.dtf)) return;
    if (!ccd_f32(A, B, a.dtf)) return;
    if (!(fminf(A.x, B.x) < a.hi)) return;          // ownership (:296)
    if (!ccd_f64(A, B, a.dt)) return;
    const unsigned long long slot = atomicAdd(a.n_hits, 1ull);
    if ((long long)slot < a.cap) a.hits[slot] = Hit{o, ab, bb};
}

// A warp owns BP_CHUNK consecutive candidates of the flattened space and
// walks them 32 at a time, lane l taking candidate base + l: the partners'
// records of a step are consecutive (coalesced), the first body is shared
// by the lanes of a segment (broadcast). Lane 0 finds the chunk's first
// segment by binary search; every lane then moves forward through the
// segment starts as its index grows.
__global__ void __launch_bounds__(BP_NT) k_candidates(const CandArgs a) {
    const int lane = threadIdx.x & 31;
    const long long chunks = (a.total + BP_CHUNK - 1) / BP_CHUNK;
    const long long na = a.n_seg / 5;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = warp0; c < chunks; c += warps) {
        const long long base = c * BP_CHUNK;
        const long long end = min(base + BP_CHUNK, a.total);
        long long s0 = 0;
        if (lane == 0) s0 = find_segment(a.seg_start, a.n_seg, base);
        long long s = __shfl_sync(0xffffffffu, s0, 0);
        long long cur = -1;
        int o = 0;
        unsigned ab = 0;
        long long col0 = 0;
        Body A{0.f, 0.f, 0.f, 0.f, 0.f};
        for (long long idx = base + lane; idx < end; idx += 32) {
            while (a.seg_start[s + 1] <= idx) ++s;
            if (s != cur) {
                cur = s;
                o = (int)(s / na);
                const long long r = s - (long long)o * na;
                ab = a.ai[r];
                A = Body{a.x[ab], a.y[ab], a.vx[ab], a.vy[ab], a.rr[ab]};
                col0 = a.seg_lo[s] - a.seg_start[s];
            }
            const long long j = col0 + idx;
            test_pair(a, o, ab, A, a.rec2[j], a.rec[j]);
        }
    }
}

}  // namespace

extern "C" int sss_broadphase(sss_ctx* ctx, const float* x, const float* y, const float* vx, const float* vy,
                              const float* rr, const unsigned char* is_ast, const unsigned char* vis, int64_t n,
                              double dt_y, double h, double halo, float lo, float hi, int* out_hits,
                              int64_t capacity, int64_t* n_hits, int64_t* n_cand, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!n_hits || !n_cand) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count pointer");
    *n_hits = 0;
    *n_cand = 0;
    if (n < 0 || capacity < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n > 0 && (!x || !y || !vx || !vy || !rr || !is_ast || !vis))
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL input");
    if (capacity > 0 && !out_hits) return sss_set_err(ctx, SSS_ERR_ARG, "NULL output");
    if (n >= ((int64_t)1 << 31)) return sss_set_err(ctx, SSS_ERR_ARG, "too many bodies");
    if (!(h > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "cell size h must be > 0");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (n < 2) return SSS_OK;
    const float hi_halo = hi + (float)halo;      // f32, as `self.hi + cp.float32(halo)`

    // scratch layout (long long units)
    const long long tiles = (n + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    const long long nn = n;
    size_t off = 0;
    auto take = [&](size_t elems) { const size_t o = off; off += (elems + 31) & ~(size_t)31; return o; };
    const size_t o_counts = take(tiles + 1);
    const size_t o_scan = take(sss_dev::scan_scratch(5 * nn + 1) + sss_dev::radix_scratch(nn));
    const size_t o_cx = take(nn), o_cy = take(nn);
    const size_t o_k0 = take(nn), o_k1 = take(nn);
    const size_t o_v = take(nn);                  // v0 + v1 (unsigned, 2 per long long)
    const size_t o_ai = take((nn + 1) / 2 + 1);
    const size_t o_seglo = take(5 * nn), o_segst = take(5 * nn + 1);
    const size_t o_rec = take(2 * nn), o_rec2 = take(nn);      // float4 and uint2 per alive body
    const size_t o_nh = take(1);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off * sizeof(long long), &scr);
    if (rc) return rc;
    long long* S = (long long*)scr;
    long long* counts = S + o_counts;
    long long* scan_tmp = S + o_scan;
    long long* cx = S + o_cx;
    long long* cy = S + o_cy;
    unsigned long long* k0 = (unsigned long long*)(S + o_k0);
    unsigned long long* k1 = (unsigned long long*)(S + o_k1);
    unsigned* v0 = (unsigned*)(S + o_v);
    unsigned* v1 = v0 + nn;
    unsigned* ai = (unsigned*)(S + o_ai);
    long long* seg_lo = S + o_seglo;
    long long* seg_st = S + o_segst;
    float4* rec = (float4*)(S + o_rec);
    uint2* rec2 = (uint2*)(S + o_rec2);
    unsigned long long* d_nh = (unsigned long long*)(S + o_nh);

    // 1) alive compaction (ascending body order) + cells + keys
    k_alive_count<<<(unsigned)tiles, BP_NT, 0, s>>>(is_ast, vis, x, nn, lo, hi_halo, counts);
    sss_dev::k_scan_sums<<<1, sss_dev::SCAN_NT, 0, s>>>(counts, tiles);
    long long na = 0;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&na, counts + tiles, sizeof(long long), cudaMemcpyDeviceToHost, s));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    if (na < 2) return SSS_OK;
    k_alive_scatter<<<(unsigned)tiles, BP_NT, 0, s>>>(is_ast, vis, x, y, nn, lo, hi_halo, h, counts, ai, cx, cy,
                                                       k0, v0);
    SSS_LAUNCH_CHECK(ctx, "k_alive_scatter");
    // 2) stable sort of the keys (ascending signed order)
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(k0, v0, k1, v1, na, scan_tmp, s));
    k_sorted_records<<<(unsigned)((na + 255) / 256), 256, 0, s>>>(x, y, vx, vy, rr, ai, v0, na, rec, rec2);
    SSS_LAUNCH_CHECK(ctx, "k_sorted_records");
    // 3) equal-key range of every (offset, body)
    const long long nseg = 5 * na;
    k_ranges<<<(unsigned)((nseg + 255) / 256), 256, 0, s>>>(cx, cy, na, k0, seg_lo, seg_st);
    SSS_LAUNCH_CHECK(ctx, "k_ranges");
    // 4) candidate offsets
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(seg_st, seg_st, nseg, scan_tmp, s));
    const long long stiles = (nseg + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    long long total = 0;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&total, scan_tmp + stiles, sizeof(long long), cudaMemcpyDeviceToHost, s));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(seg_st + nseg, scan_tmp + stiles, sizeof(long long), cudaMemcpyDeviceToDevice,
                                      s));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(d_nh, 0, sizeof(unsigned long long), s));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    *n_cand = total;
    if (total == 0) return SSS_OK;
    // 5) fused candidate walk + tests
    CandArgs ca;
    ca.x = x; ca.y = y; ca.vx = vx; ca.vy = vy; ca.rr = rr;
    ca.ai = ai;
    ca.rec = rec;
    ca.rec2 = rec2;
    ca.seg_lo = seg_lo;
    ca.seg_start = seg_st;
    ca.n_seg = nseg;
    ca.total = total;
    ca.dtf = (float)dt_y;
    ca.dt = dt_y;
    ca.hi = hi;
    ca.hits = (Hit*)out_hits;
    ca.cap = capacity;
    ca.n_hits = d_nh;
    const long long chunks = (total + BP_CHUNK - 1) / BP_CHUNK;
    long long blocks = (chunks + BP_NT / 32 - 1) / (BP_NT / 32);
    const long long max_blocks = (long long)ctx->num_sms * 32;
    if (blocks > max_blocks) blocks = max_blocks;
    k_candidates<<<(unsigned)blocks, BP_NT, 0, s>>>(ca);
    SSS_LAUNCH_CHECK(ctx, "k_candidates");
    unsigned long long nh = 0;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&nh, d_nh, sizeof(nh), cudaMemcpyDeviceToHost, s));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    *n_hits = (int64_t)nh;
    if ((long long)nh > capacity)
        return sss_set_err(ctx, SSS_ERR_CAPACITY, "hit buffer holds %lld, %llu hits found", (long long)capacity, nh);
    return SSS_OK;
}
