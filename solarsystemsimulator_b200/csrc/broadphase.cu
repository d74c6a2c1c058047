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
// The candidate list is never materialised: the bodies are sorted by cell
// key and, inside a cell, by sub-cell, and split into runs of one cell; a run
// and a neighbour offset give a block of candidates (the run's bodies x the
// bodies with the offset cell's key), counted exactly and cut into tiles of
// 32 run bodies x up to 992 partners. A warp skips each aligned chunk of 32
// partners whose bounding box is provably out of reach of the run bodies' box
// and streams the others as broadcast loads from records stored in sorted
// order. Hits are appended; sss_broadphase_order sorts them by (offset, a, b)
// on the device, which is the reference's output order.

#include "devscan.cuh"

namespace {

constexpr int BP_NT = 256;

// The call's scalars, in device memory: the kernels read them there, so one
// captured graph of the pipeline serves every call of the same size.
struct BpParams {
    float lo, hi_halo, hi, dtf;
    double h, dt;
};

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
                                                       const float* __restrict__ x, long long n,
                                                       const BpParams* __restrict__ P,
                                                       long long* __restrict__ counts,
                                                       unsigned long long* __restrict__ kmin) {
    const float lo = P->lo, hi_halo = P->hi_halo;
    const long long base = (long long)blockIdx.x * sss_dev::SCAN_TILE;
    if (blockIdx.x == 0 && threadIdx.x == 0) {                   // the alive scatter narrows them
        kmin[0] = ~0ull;
        kmin[1] = 0ull;
    }
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
                                                         long long n, const BpParams* __restrict__ P,
                                                         const long long* __restrict__ offs,
                                                         unsigned* __restrict__ ai, long long* __restrict__ cx,
                                                         long long* __restrict__ cy,
                                                         unsigned long long* __restrict__ skey,
                                                         unsigned* __restrict__ sval,
                                                         unsigned long long* __restrict__ kmin) {   // [min, max]
    const float lo = P->lo, hi_halo = P->hi_halo;
    const double h = P->h;
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
    unsigned long long kl = ~0ull, kh = 0ull;                       // this thread's smallest and largest key
    for (int k = 0; k < sss_dev::SCAN_ITEMS; ++k) {
        if (!f[k]) continue;
        const long long i = base + (long long)threadIdx.x * sss_dev::SCAN_ITEMS + k;
        const long long ix = (long long)floor(__ddiv_rn((double)x[i], h));
        const long long iy = (long long)floor(__ddiv_rn((double)y[i], h));
        ai[r] = (unsigned)i;
        cx[r] = ix;
        cy[r] = iy;
        // signed int64 order as unsigned: flip the sign bit
        const unsigned long long kk = (unsigned long long)cell_key(ix, iy) ^ 0x8000000000000000ull;
        skey[r] = kk;
        sval[r] = (unsigned)r;
        kl = kk < kl ? kk : kl;
        kh = kk > kh ? kk : kh;
        ++r;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, kl, o);
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, kh, o);
        kl = v < kl ? v : kl;
        kh = w > kh ? w : kh;
    }
    if ((threadIdx.x & 31) == 0 && kl <= kh) {
        atomicMin(&kmin[0], kl);
        atomicMax(&kmin[1], kh);
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
                                 const unsigned* __restrict__ order, const long long* __restrict__ d_na,
                                 float4* __restrict__ rec, uint2* __restrict__ rec2) {
    const long long pos = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= *d_na) return;
    const unsigned b = ai[order[pos]];
    rec[pos] = make_float4(x[b], y[b], vx[b], vy[b]);
    rec2[pos] = make_uint2(__float_as_uint(rr[b]), b);
}

struct TestParams {
    float dtf, hi;
    double dt;
    Hit* hits;
    long long cap;
    unsigned long long* n_hits;
};

// The last s in [0, n_seg) with start[s] <= idx (start non-decreasing,
// start[0] = 0 <= idx), searched by the whole warp: each round the 32 lanes
// probe 32 evenly spaced entries of [lo, hi) and the ballot's highest set
// bit narrows the range 32-fold (4 rounds of loads for a million entries
// instead of 20 dependent ones). Warp-uniform; every lane returns s.
__device__ __forceinline__ long long find_segment(const long long* start, long long n_seg, long long idx, int lane) {
    long long lo = 0, hi = n_seg;     // start[lo] <= idx; s < hi
    while (hi - lo > 1) {
        const long long step = (hi - lo + 31) / 32;
        const long long m = lo + (long long)lane * step;
        const bool le = m < hi && start[m] <= idx;
        const unsigned b = __ballot_sync(0xffffffffu, le);     // a prefix of the lanes, lane 0 included
        lo += (long long)(31 - __clz(b)) * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// ownership and the f64 recheck after the f32 test, then the append (film_producer.py:241-314)
__device__ __forceinline__ void test_exact(const TestParams& a, int o, unsigned ab, const Body& A, unsigned bb,
                                           const Body& B) {
    if (!ccd_f32(A, B, a.dtf)) return;
    if (!(fminf(A.x, B.x) < a.hi)) return;          // ownership (:296)
    if (!ccd_f64(A, B, a.dt)) return;
    const unsigned long long slot = atomicAdd(a.n_hits, 1ull);
    if ((long long)slot < a.cap) a.hits[slot] = Hit{o, ab, bb};
}

// Position inside the cell: a 12-bit Morton code of the 64 x 64 sub-cell,
// the secondary sort key, so that consecutive bodies of a run (and of a
// partner range) lie close together and their bounding boxes are small.
__device__ __forceinline__ unsigned spread2(unsigned v) {
    v &= 0x3Fu;
    v = (v | (v << 4)) & 0x0F0Fu;
    v = (v | (v << 2)) & 0x3333u;
    v = (v | (v << 1)) & 0x5555u;
    return v;
}

__global__ void k_sub_keys(const float* __restrict__ x, const float* __restrict__ y, const unsigned* __restrict__ ai,
                           const long long* __restrict__ cx, const long long* __restrict__ cy,
                           const long long* __restrict__ d_na, long long n, const BpParams* __restrict__ P,
                           unsigned long long* __restrict__ sk, unsigned* __restrict__ sv) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const double h = P->h;
    if (r >= *d_na) {                                              // padding up to n: sorts after every row
        sk[r] = 0xFFFull;
        sv[r] = (unsigned)r;
        return;
    }
    const unsigned b = ai[r];
    const double fx = __ddiv_rn((double)x[b], h) - (double)cx[r];
    const double fy = __ddiv_rn((double)y[b], h) - (double)cy[r];
    const int ix = fx >= 0.0 ? min((int)(fx * 64.0), 63) : 0;      // NaN and below: sub-cell 0
    const int iy = fy >= 0.0 ? min((int)(fy * 64.0), 63) : 0;
    sk[r] = spread2((unsigned)ix) | (spread2((unsigned)iy) << 1);
    sv[r] = (unsigned)r;
}

// Cell keys in sub-cell order, as offsets from the smallest alive key
// (kmin = [smallest, largest]): the same order and the same equal groups,
// and the high digits of a compact key range are zero, so the radix sort
// copies those passes instead of ranking them. Padding rows take the largest
// offset: they come after every alive row in this order, so the stable sort
// keeps them last.
__global__ void k_gather_keys(const unsigned long long* __restrict__ rowkey, const unsigned* __restrict__ order,
                              const long long* __restrict__ d_na, long long n,
                              const unsigned long long* __restrict__ kmin, unsigned long long* __restrict__ keys) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) keys[p] = (p < *d_na ? rowkey[order[p]] : kmin[1]) - kmin[0];
}

// Bounding box of every aligned chunk of 32 sorted records: x, y, vx, vy
// ranges and the largest radius (NaN when a radius is NaN).
struct ChunkBox {
    float4 pos;   // xmin, xmax, ymin, ymax
    float4 vel;   // vxmin, vxmax, vymin, vymax
    float4 rad;   // rrmax, -, -, -
};

__device__ __forceinline__ float nan_max(float a, float b) { return (b > a || b != b) ? b : a; }

__global__ void k_chunk_boxes(const float4* __restrict__ rec, const uint2* __restrict__ rec2,
                              const long long* __restrict__ d_na, ChunkBox* __restrict__ boxes) {
    const int lane = threadIdx.x & 31;
    const long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long na = *d_na;
    const long long nc = (na + 31) / 32;
    if (c >= nc) return;
    const long long j = c * 32 + lane;
    float4 v = make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
    float4 w = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
    float r = 0.0f;
    if (j < na) {
        const float4 q = rec[j];
        v = q;
        w = q;
        r = __uint_as_float(rec2[j].x);
    }
    for (int d = 16; d; d >>= 1) {
        v.x = fminf(v.x, __shfl_xor_sync(0xffffffffu, v.x, d));
        v.y = fminf(v.y, __shfl_xor_sync(0xffffffffu, v.y, d));
        v.z = fminf(v.z, __shfl_xor_sync(0xffffffffu, v.z, d));
        v.w = fminf(v.w, __shfl_xor_sync(0xffffffffu, v.w, d));
        w.x = fmaxf(w.x, __shfl_xor_sync(0xffffffffu, w.x, d));
        w.y = fmaxf(w.y, __shfl_xor_sync(0xffffffffu, w.y, d));
        w.z = fmaxf(w.z, __shfl_xor_sync(0xffffffffu, w.z, d));
        w.w = fmaxf(w.w, __shfl_xor_sync(0xffffffffu, w.w, d));
        r = nan_max(r, __shfl_xor_sync(0xffffffffu, r, d));
    }
    if (lane == 0) {
        boxes[c].pos = make_float4(v.x, w.x, v.y, w.y);
        boxes[c].vel = make_float4(v.z, w.z, v.w, w.w);
        boxes[c].rad = make_float4(r, 0.0f, 0.0f, 0.0f);
    }
}

// Cell runs: consecutive sorted positions whose bodies lie in the same cell
// (the bodies of two cells with colliding keys interleave in the stable key
// order; each stretch of one cell is its own run). All bodies of a run have,
// per neighbour offset, the same partner range (the bodies whose key is the
// offset cell's key), so the candidates of (run, offset) form a block of
// run length x range length pairs. The candidate set, and with it the hit
// set, is the reference's; the order of the hits is restored by sorting them
// by (offset, a, b).
__global__ void k_run_flags(const long long* __restrict__ cx, const long long* __restrict__ cy,
                            const unsigned* __restrict__ order, const long long* __restrict__ d_na, long long n,
                            long long* __restrict__ flags) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (p >= *d_na) {                                              // padding: no runs
        flags[p] = 0;
        return;
    }
    bool start = p == 0;
    if (!start) {
        const unsigned r = order[p], q = order[p - 1];
        start = cx[r] != cx[q] || cy[r] != cy[q];
    }
    flags[p] = start ? 1 : 0;
}

__global__ void k_run_starts(const long long* __restrict__ flags, const long long* __restrict__ pos,
                             const long long* __restrict__ d_na, long long* __restrict__ run_start) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < *d_na && flags[p]) run_start[pos[p]] = p;
}

constexpr int TILE_B = 992;       // partners per tile (at most 32 aligned chunks of 32); 32 run bodies per tile

// Item t = o * n_run + q: run q against the partner range of offset o (its
// first position and length), its tile count, and the candidates summed per
// block into n_cand. Launched over an upper bound of items; those past
// 5 n_run get no tiles.
__global__ void __launch_bounds__(256) k_items(const long long* __restrict__ cx, const long long* __restrict__ cy,
                                               const unsigned* __restrict__ order,
                                               const unsigned long long* __restrict__ ks,
                                               const unsigned long long* __restrict__ kmin,
                                               const long long* __restrict__ d_na,
                                               const long long* __restrict__ run_start,
                                               const long long* __restrict__ d_nrun, long long max_items,
                                               long long* __restrict__ item_b0, long long* __restrict__ item_nb,
                                               long long* __restrict__ tiles, unsigned long long* __restrict__ n_cand) {
    __shared__ unsigned long long bs[8];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long na = *d_na, n_run = *d_nrun;
    unsigned long long cand = 0;
    if (t < max_items && t >= 5 * n_run) tiles[t] = 0;
    if (t < 5 * n_run) {
        const int o = (int)(t / n_run);
        const long long q = t - (long long)o * n_run;
        const long long p0 = run_start[q], p1 = q + 1 < n_run ? run_start[q + 1] : na;
        const unsigned r = order[p0];
        // (a key below the smallest wraps to a value no alive key has)
        const unsigned long long k2 =
            ((unsigned long long)cell_key(cx[r] + c_off[o][0], cy[r] + c_off[o][1]) ^ 0x8000000000000000ull) - kmin[0];
        const long long lo = lower_bound(ks, na, k2);
        const long long nb = upper_bound(ks, na, k2) - lo;
        item_b0[t] = lo;
        item_nb[t] = nb;
        tiles[t] = ((p1 - p0 + 31) / 32) * ((nb + TILE_B - 1) / TILE_B);
        cand = (unsigned long long)(p1 - p0) * (unsigned long long)nb;
    }
    for (int d = 16; d; d >>= 1) cand += __shfl_down_sync(0xffffffffu, cand, d);
    if ((threadIdx.x & 31) == 0) bs[threadIdx.x >> 5] = cand;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0;
        for (int w = 0; w < 8; ++w) sum += bs[w];
        if (sum) atomicAdd(n_cand, sum);
    }
}

struct TileArgs {
    const float4* rec;           // sorted position -> (x, y, vx, vy)
    const uint2* rec2;           // sorted position -> (rr bits, body)
    const long long* run_start;  // [n_run]
    const long long* item_b0;    // [5 n_run]
    const long long* item_nb;    // [5 n_run]
    const long long* tile_start; // [5 n_run + 1] exclusive prefix of the tile counts
    const unsigned long long* ks; // sorted keys
    const ChunkBox* boxes;       // [ceil(na / 32)] boxes of the aligned chunks of 32 records
    const long long* na;         // alive bodies, runs and tiles (device counts)
    const long long* n_run;
    const long long* n_tiles;
    const BpParams* P;           // dtf, dt, hi of tp come from here
    unsigned long long* tile_ctr; // the next tile to hand out (zero before the launch)
    TestParams tp;
};

constexpr int TILE_GRAB = 1;      // tiles a warp takes from the counter at a time (measured: 1 0.61 ms,
                                  // 2 0.63, 4 0.66, 8 0.79 per device call on the 200k-asteroid clouds)

__device__ __forceinline__ float warp_max(float v) {
    for (int d = 16; d; d >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}
__device__ __forceinline__ float warp_min(float v) {
    for (int d = 16; d; d >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}

// Pairs that provably fail the f32 test are skipped before it. That test
// evaluates the closest approach |dp + dv t| at some t in [-dt, dt], from
// the rounded dp = B - A, dv (the same subtractions). For every t,
// |dp + dv t| >= |dp x dv| / |dv|, the distance of the relative motion's
// line (dp x dv = dpx dvy - dpy dvx). So a pair is skipped when
//   (|dp x dv| - E)^2 > 4.01 rs^2 |dv|^2,  rs = (rr_a + 1e-6) + rr_b,
// i.e. its line passes farther than 2 rs. E bounds the f32 error of the
// cross product: with |dpx|, |dpy| <= P and |dvx|, |dvy| <= V over the tile,
// |dpx dvy| + |dpy dvx| <= 2 P V and the error is below 2^-22 of that;
// E = 2 EPS_CROSS P V with EPS_CROSS = 4e-6 (>= 32 ulp). The skip is taken
// only when P and V dt stay below 0.5 AU over the whole tile: then the f32
// test's own rounding moves its distance by less than 1e-7 AU, while
// rs >= 1e-6 AU, and 4.01 instead of 4 covers the rounding of the
// comparison and of rs (a few ulp). A skipped pair can never pass the f32
// test: the skips change no result, only the work.
constexpr float EPS_CROSS = 4.0e-6f;
constexpr int QCAP = 64;          // queued pairs per warp (flushed at 32)

// Queue of pairs the line test could not skip (per warp, in shared memory):
// push the lanes' pairs of this step, and once 32 are queued test them
// exactly, one per lane (the run body fetched from its lane by shuffles).
struct PairQueue {
    int* j;
    unsigned char* l;
    int cnt;
};

__device__ __forceinline__ void queue_flush(PairQueue& q, int n, const TileArgs& a, int o, const Body& A,
                                            unsigned ab, int lane) {
    const int src = lane < n ? q.l[lane] : 0;
    const int jj = lane < n ? q.j[lane] : 0;
    const Body As{__shfl_sync(0xffffffffu, A.x, src), __shfl_sync(0xffffffffu, A.y, src),
                  __shfl_sync(0xffffffffu, A.vx, src), __shfl_sync(0xffffffffu, A.vy, src),
                  __shfl_sync(0xffffffffu, A.rr, src)};
    const unsigned abs_ = __shfl_sync(0xffffffffu, ab, src);
    if (lane < n) {
        const float4 bv = a.rec[jj];
        const uint2 bw = a.rec2[jj];
        test_exact(a.tp, o, abs_, As, bw.y, Body{bv.x, bv.y, bv.z, bv.w, __uint_as_float(bw.x)});
    }
    __syncwarp();
}

__device__ __forceinline__ void queue_push(PairQueue& q, unsigned m, bool need, int j, const TileArgs& a, int o,
                                           const Body& A, unsigned ab, int lane) {
    if (need) {
        const int at = q.cnt + __popc(m & ((1u << lane) - 1u));
        q.j[at] = j;
        q.l[at] = (unsigned char)lane;
    }
    q.cnt += __popc(m);
    __syncwarp();
    if (q.cnt >= 32) {
        queue_flush(q, 32, a, o, A, ab, lane);
        if (lane < q.cnt - 32) {
            q.j[lane] = q.j[lane + 32];
            q.l[lane] = q.l[lane + 32];
        }
        q.cnt -= 32;
        __syncwarp();
    }
}

// The partners [j0, j0 + nj) of one surviving chunk against the lane's run
// body (valid = false: the lane has none). Keep rule on body indices:
// MODE 0: offset (0, 0), keep a < b; MODE 1: another offset whose key
// differs from the run's own, all pairs kept (the two ranges are disjoint);
// MODE 2: another offset whose cell key equals the run's own (a hash
// collision), keep a != b. The line test (see above) uses the chunk's
// largest radius (kl = 4.01 (rr_a + 1e-6 + rr_max)^2), which can only make it
// skip less; it is written as c |c| > kl dv^2 with c = |dp x dv| - E, false
// for c <= 0.
template <int MODE>
__device__ __forceinline__ void span_walk(const TileArgs& a, int o, const Body& A, unsigned ab, bool valid,
                                          long long j0, int nj, float E, float kl, bool skip_ok, PairQueue& q,
                                          int lane) {
    const float4* rp = a.rec + j0;
    const uint2* rp2 = a.rec2 + j0;
    auto keep_of = [&](int k) {
        if (MODE == 1) return true;
        const unsigned bb = __ldg(&rp2[k].y);
        return MODE == 0 ? ab < bb : ab != bb;
    };
    if (!skip_ok) {                                    // no skips in this chunk: every kept pair is tested
        for (int k = 0; k < nj; ++k) {
            const bool need = valid && keep_of(k);
            const unsigned m = __ballot_sync(0xffffffffu, need);
            if (m) queue_push(q, m, need, (int)(j0 + k), a, o, A, ab, lane);
        }
        return;
    }
    int k = 0;
    for (; k + 4 <= nj; k += 4) {
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = __ldg(rp + k + u);
        bool need[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float dpx = v[u].x - A.x, dpy = v[u].y - A.y;
            const float dvx = v[u].z - A.vx, dvy = v[u].w - A.vy;
            const float c = fabsf(dpx * dvy - dpy * dvx) - E;
            need[u] = valid && !(c * fabsf(c) > kl * (dvx * dvx + dvy * dvy)) && keep_of(k + u);
        }
        const unsigned any = __ballot_sync(0xffffffffu, need[0] || need[1] || need[2] || need[3]);
        if (any) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const unsigned m = __ballot_sync(0xffffffffu, need[u]);
                if (m) queue_push(q, m, need[u], (int)(j0 + k + u), a, o, A, ab, lane);
            }
        }
    }
    for (; k < nj; ++k) {
        const float4 v = __ldg(rp + k);
        const float dpx = v.x - A.x, dpy = v.y - A.y;
        const float dvx = v.z - A.vx, dvy = v.w - A.vy;
        const float c = fabsf(dpx * dvy - dpy * dvx) - E;
        const bool need = valid && !(c * fabsf(c) > kl * (dvx * dvx + dvy * dvy)) && keep_of(k);
        const unsigned m = __ballot_sync(0xffffffffu, need);
        if (m) queue_push(q, m, need, (int)(j0 + k), a, o, A, ab, lane);
    }
}

// A warp takes a contiguous range of tiles (one binary search per warp,
// then forward). Per tile: lane l holds run body p0 + 32 i + l; the tile's
// partners span at most 32 aligned chunks of 32 records, and lane c tests
// chunk c against the box of the run bodies: the chunk is skipped when every
// pair of it is provably apart (below); the warp walks the surviving chunks
// one by one, streaming their partners as broadcast loads through the keep
// rule and the line test, and queues the pairs it cannot skip.
//
// Chunk skip: over all pairs of the run bodies and the chunk, |dp| is at
// least the distance d of the two boxes and every (|dvx| + |dvy|) dt + rs is
// at most reach = (Vx + Vy) dt + (rr_a,max + 1e-6 + rr_b,max) (Vx, Vy the
// largest velocity differences of the boxes). If d > 2 reach, each pair has
// |dp| > 2 ((|dvx| + |dvy|) dt + rs), so its closest approach over t in
// [-dt, dt] exceeds 2 rs: the f32 test rejects it (its own rounding below
// 1e-7 AU while the boxes' extents P and V dt stay below 0.5 AU, rs >= 1e-6
// AU); 4.01 for 4 covers the rounding of the box arithmetic.
__global__ void __launch_bounds__(BP_NT, 3) k_tiles(const TileArgs a_in) {
    TileArgs a = a_in;
    a.tp.dtf = a_in.P->dtf;
    a.tp.dt = a_in.P->dt;
    a.tp.hi = a_in.P->hi;
    __shared__ int q_j[BP_NT / 32][QCAP];
    __shared__ unsigned char q_l[BP_NT / 32][QCAP];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    PairQueue q{q_j[wib], q_l[wib], 0};
    const long long na = *a.na, n_run = *a.n_run, n_tiles = *a.n_tiles;
    const long long n_items = 5 * n_run;
    const float dtf = a.tp.dtf;
    // the tiles' costs differ by orders of magnitude (culled chunks against
    // dense ones), so the warps take them one at a time from a counter
    // instead of fixed shares
    for (;;) {
        long long g0 = 0;
        if (lane == 0) g0 = (long long)atomicAdd(a.tile_ctr, (unsigned long long)TILE_GRAB);
        const long long tb = __shfl_sync(0xffffffffu, g0, 0);
        if (tb >= n_tiles) break;
        const long long te = min(tb + (long long)TILE_GRAB, n_tiles);
        long long t = find_segment(a.tile_start, n_items, tb, lane);
        long long t_start = a.tile_start[t], t_end = a.tile_start[t + 1];
        for (long long tid = tb; tid < te; ++tid) {
            while (t_end <= tid) {
                ++t;
                t_start = t_end;
                t_end = a.tile_start[t + 1];
            }
            const int o = (int)(t / n_run);
            const long long qr = t - (long long)o * n_run;
            const long long p0 = a.run_start[qr], p1 = qr + 1 < n_run ? a.run_start[qr + 1] : na;
            const long long b0 = a.item_b0[t], nb = a.item_nb[t];
            const long long n_bt = (nb + TILE_B - 1) / TILE_B;
            const long long local = tid - t_start;
            const long long ai = local / n_bt, bi = local - ai * n_bt;
            const long long pa = p0 + ai * 32 + lane;
            const bool valid = pa < p1;
            Body A{0.f, 0.f, 0.f, 0.f, 0.f};
            unsigned ab = 0;
            if (valid) {
                const float4 v = a.rec[pa];
                const uint2 w = a.rec2[pa];
                A = Body{v.x, v.y, v.z, v.w, __uint_as_float(w.x)};
                ab = w.y;
            }
            const float ax0 = warp_min(valid ? A.x : INFINITY), ax1 = warp_max(valid ? A.x : -INFINITY);
            const float ay0 = warp_min(valid ? A.y : INFINITY), ay1 = warp_max(valid ? A.y : -INFINITY);
            const float au0 = warp_min(valid ? A.vx : INFINITY), au1 = warp_max(valid ? A.vx : -INFINITY);
            const float aw0 = warp_min(valid ? A.vy : INFINITY), aw1 = warp_max(valid ? A.vy : -INFINITY);
            float arr = valid ? A.rr : 0.0f;
            for (int d = 16; d; d >>= 1) arr = nan_max(arr, __shfl_xor_sync(0xffffffffu, arr, d));
            const long long jb = b0 + bi * TILE_B;
            const long long je = min(jb + TILE_B, b0 + nb);
            const long long c0 = jb >> 5;
            const int nch = (int)(((je - 1) >> 5) - c0 + 1);
            // lane c: chunk c0 + c
            bool near = false;
            float Pc = 0.0f, Vc = 0.0f, brr = 0.0f;
            if (lane < nch) {
                const ChunkBox bx = a.boxes[c0 + lane];
                const float dxb = fmaxf(0.0f, fmaxf(bx.pos.x - ax1, ax0 - bx.pos.y));
                const float dyb = fmaxf(0.0f, fmaxf(bx.pos.z - ay1, ay0 - bx.pos.w));
                const float Vx = fmaxf(bx.vel.y - au0, au1 - bx.vel.x), Vy = fmaxf(bx.vel.w - aw0, aw1 - bx.vel.z);
                Pc = fmaxf(fmaxf(bx.pos.y - ax0, ax1 - bx.pos.x), fmaxf(bx.pos.w - ay0, ay1 - bx.pos.z)) * 1.0001f;
                Vc = fmaxf(Vx, Vy) * 1.0001f;
                brr = bx.rad.x;
                const float reach = (Vx + Vy) * 1.0001f * dtf + ((arr + 1e-6f) + brr);
                const float d2 = dxb * dxb + dyb * dyb;
                const bool far = Pc < 0.5f && Vc * dtf < 0.5f && reach < 1.0f && d2 > 4.01f * reach * reach;
                near = !far;
            }
            unsigned nm = __ballot_sync(0xffffffffu, near);
            const int mode = o == 0 ? 0 : (a.ks[b0] != a.ks[p0] ? 1 : 2);
            const float rsa = A.rr + 1e-6f;
            while (nm) {
                const int c = __ffs(nm) - 1;
                nm &= nm - 1;
                const float P = __shfl_sync(0xffffffffu, Pc, c), V = __shfl_sync(0xffffffffu, Vc, c);
                const float br = __shfl_sync(0xffffffffu, brr, c);
                // a NaN radius or an unbounded box: no line-test skips in the chunk (warp-uniform;
                // NaN coordinates need nothing here, as their line test never skips)
                const bool skip_ok =
                    __all_sync(0xffffffffu, P < 0.5f && V * dtf < 0.5f && br == br && (!valid || A.rr == A.rr));
                const float E = 2.0f * EPS_CROSS * P * V;
                const float rs = rsa + br;
                const float kl = 4.01f * rs * rs;
                const long long cs = (c0 + c) << 5;
                const long long js = max(cs, jb), jn = min(cs + 32, je);
                if (mode == 0) span_walk<0>(a, o, A, ab, valid, js, (int)(jn - js), E, kl, skip_ok, q, lane);
                else if (mode == 1) span_walk<1>(a, o, A, ab, valid, js, (int)(jn - js), E, kl, skip_ok, q, lane);
                else span_walk<2>(a, o, A, ab, valid, js, (int)(jn - js), E, kl, skip_ok, q, lane);
            }
            if (q.cnt > 0) {                               // the rest of the tile's queue
                queue_flush(q, q.cnt, a, o, A, ab, lane);
                q.cnt = 0;
            }
        }
    }
}

// Hit order of the reference's output, (offset, a, b) ascending, as one
// 64-bit key: offset (3 bits) above a and b (B bits each, a, b < 2^B).
__global__ void k_hit_keys(const Hit* __restrict__ h, long long k, int B, unsigned long long* __restrict__ keys,
                           unsigned* __restrict__ vals) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const Hit v = h[i];
    keys[i] = ((unsigned long long)(unsigned)v.o << (2 * B)) | ((unsigned long long)v.a << B) | v.b;
    vals[i] = (unsigned)i;
}

__global__ void k_hit_gather(const Hit* __restrict__ in, const unsigned* __restrict__ order, long long k,
                             Hit* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) out[i] = in[order[i]];
}

// The call's inputs into the staging arrays the captured pipeline reads.
__global__ void k_bp_stage(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ vx,
                           const float* __restrict__ vy, const float* __restrict__ rr,
                           const unsigned char* __restrict__ is_ast, const unsigned char* __restrict__ vis,
                           long long n, float* __restrict__ f5, unsigned char* __restrict__ u2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f5[i] = x[i];
    f5[n + i] = y[i];
    f5[2 * n + i] = vx[i];
    f5[3 * n + i] = vy[i];
    f5[4 * n + i] = rr[i];
    u2[i] = is_ast[i];
    u2[n + i] = vis[i];
}

}  // namespace

// One instantiated graph of the broadphase pipeline per context: the launch
// sequence depends only on n, the hit capacity and the scratch address, so a
// call of the same size replays it (one graph launch instead of ~30 launches
// and clears). Counts come back through pinned host memory.
struct sss_bp_graph {
    long long n = -1, cap = -1;
    void* base = nullptr;
    cudaGraphExec_t exec = nullptr;
    BpParams* h_par = nullptr;               // pinned
    unsigned long long* h_cnt = nullptr;     // pinned: hits, candidates, alive
};

void sss_bp_graph_free(sss_bp_graph* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->h_par) cudaFreeHost(g->h_par);
    if (g->h_cnt) cudaFreeHost(g->h_cnt);
    delete g;
}

namespace {

// Device pointers of one call's pipeline (all inside the context scratch).
struct BpBufs {
    const float *x, *y, *vx, *vy, *rr;
    const unsigned char *is_ast, *vis;
    const BpParams* P;
    long long* counts;
    long long* scan_tmp;
    long long *cx, *cy;
    unsigned long long *k0, *k1;
    unsigned *v0, *v1, *ai;
    long long *flags, *pos, *run_start, *item_b0, *item_nb, *tile_st;
    float4* rec;
    uint2* rec2;
    unsigned long long* rowkey;
    ChunkBox* boxes;
    unsigned long long* d_nh;   // hits, candidates, smallest and largest alive cell key, tile counter
    Hit* hits;
};

// The launch sequence of one call on stream s (captured into a graph). Every
// size after the alive count stays on the device: the launches are sized for
// n bodies (5 n items, a persistent tile grid) and read the counts there.
int enqueue_pipeline(sss_ctx* ctx, const BpBufs& B, long long nn, long long capacity, cudaStream_t s) {
    const long long tiles = (nn + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    // 1) alive compaction (ascending body order) + cells + keys
    k_alive_count<<<(unsigned)tiles, BP_NT, 0, s>>>(B.is_ast, B.vis, B.x, nn, B.P, B.counts, B.d_nh + 2);
    sss_dev::k_scan_sums<<<1, sss_dev::SCAN_NT, 0, s>>>(B.counts, tiles);
    const long long* d_na = B.counts + tiles;
    k_alive_scatter<<<(unsigned)tiles, BP_NT, 0, s>>>(B.is_ast, B.vis, B.x, B.y, nn, B.P, B.counts, B.ai, B.cx,
                                                       B.cy, B.rowkey, B.v0, B.d_nh + 2);
    SSS_LAUNCH_CHECK(ctx, "k_alive_scatter");
    // 2) sort by the position inside the cell, then stably by the cell key
    //    (ascending signed order): key, then sub-cell, then body order; the
    //    n - na padding entries sort last in both
    const unsigned nb_n = (unsigned)((nn + 255) / 256);
    k_sub_keys<<<nb_n, 256, 0, s>>>(B.x, B.y, B.ai, B.cx, B.cy, d_na, nn, B.P, B.k0, B.v0);
    SSS_LAUNCH_CHECK(ctx, "k_sub_keys");
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(B.k0, B.v0, B.k1, B.v1, nn, B.scan_tmp, s, ctx->d_status, 12));
    k_gather_keys<<<nb_n, 256, 0, s>>>(B.rowkey, B.v0, d_na, nn, B.d_nh + 2, B.k0);
    SSS_LAUNCH_CHECK(ctx, "k_gather_keys");
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(B.k0, B.v0, B.k1, B.v1, nn, B.scan_tmp, s, ctx->d_status));
    k_sorted_records<<<nb_n, 256, 0, s>>>(B.x, B.y, B.vx, B.vy, B.rr, B.ai, B.v0, d_na, B.rec, B.rec2);
    SSS_LAUNCH_CHECK(ctx, "k_sorted_records");
    const long long n_chunks = (nn + 31) / 32;
    k_chunk_boxes<<<(unsigned)((n_chunks * 32 + 255) / 256), 256, 0, s>>>(B.rec, B.rec2, d_na, B.boxes);
    SSS_LAUNCH_CHECK(ctx, "k_chunk_boxes");
    // 3) cell runs of the sorted order
    k_run_flags<<<nb_n, 256, 0, s>>>(B.cx, B.cy, B.v0, d_na, nn, B.flags);
    SSS_LAUNCH_CHECK(ctx, "k_run_flags");
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(B.flags, B.pos, nn, B.scan_tmp, s, ctx->d_status));
    // the run count: the scan's total, kept after the items' tile starts
    const long long ntiles_n = (nn + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    long long* d_nrun = B.tile_st + 5 * nn + 1;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(d_nrun, B.scan_tmp + ntiles_n, sizeof(long long), cudaMemcpyDeviceToDevice, s));
    k_run_starts<<<nb_n, 256, 0, s>>>(B.flags, B.pos, d_na, B.run_start);
    SSS_LAUNCH_CHECK(ctx, "k_run_starts");
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(B.d_nh, 0, 2 * sizeof(unsigned long long), s));
    // 4) (run, offset) items: partner ranges, tiles, candidates
    const long long max_items = 5 * nn;
    k_items<<<(unsigned)((max_items + 255) / 256), 256, 0, s>>>(B.cx, B.cy, B.v0, B.k0, B.d_nh + 2, d_na,
                                                                B.run_start, d_nrun,
                                                                max_items, B.item_b0, B.item_nb, B.tile_st,
                                                                B.d_nh + 1);
    SSS_LAUNCH_CHECK(ctx, "k_items");
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(B.tile_st, B.tile_st, max_items, B.scan_tmp, s, ctx->d_status));
    const long long itiles = (max_items + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    long long* d_ntiles = B.tile_st + 5 * nn + 2;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(B.tile_st + max_items, B.scan_tmp + itiles, sizeof(long long),
                                      cudaMemcpyDeviceToDevice, s));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(d_ntiles, B.scan_tmp + itiles, sizeof(long long), cudaMemcpyDeviceToDevice, s));
    // 5) tiles: keep rule + tests (a persistent grid; warps split the tiles)
    TileArgs ta;
    ta.rec = B.rec;
    ta.rec2 = B.rec2;
    ta.run_start = B.run_start;
    ta.item_b0 = B.item_b0;
    ta.item_nb = B.item_nb;
    ta.tile_start = B.tile_st;
    ta.ks = B.k0;
    ta.boxes = B.boxes;
    ta.na = d_na;
    ta.n_run = d_nrun;
    ta.n_tiles = d_ntiles;
    ta.P = B.P;
    ta.tp.dtf = 0.0f;      // from P in the kernel
    ta.tp.dt = 0.0;
    ta.tp.hi = 0.0f;
    ta.tp.hits = B.hits;
    ta.tp.cap = capacity;
    ta.tp.n_hits = B.d_nh;
    ta.tile_ctr = B.d_nh + 4;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(ta.tile_ctr, 0, sizeof(unsigned long long), s));
    k_tiles<<<(unsigned)(ctx->num_sms * 32), BP_NT, 0, s>>>(ta);
    SSS_LAUNCH_CHECK(ctx, "k_tiles");
    return SSS_OK;
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
    const size_t o_flag = take(nn), o_pos = take(nn), o_run = take(nn);
    const size_t o_ib0 = take(5 * nn), o_inb = take(5 * nn), o_tst = take(5 * nn + 3);  // + run and tile counts
    const size_t o_rec = take(2 * nn), o_rec2 = take(nn);      // float4 and uint2 per alive body
    const size_t o_rowkey = take(nn);                          // cell key per alive row
    const size_t o_box = take((nn + 31) / 32 * (sizeof(ChunkBox) / 8));
    const size_t o_nh = take(5);                               // hits, candidates, smallest and largest cell key, tile counter
    const size_t o_par = take(sizeof(BpParams) / 8 + 1);
    const size_t o_f5 = take((5 * nn + 1) / 2);                // staged x, y, vx, vy, rr (f32)
    const size_t o_u2 = take((2 * nn + 7) / 8);                // staged is_ast, vis (u8)
    const size_t o_hits = take(((size_t)capacity * sizeof(Hit) + 7) / 8);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off * sizeof(long long), &scr);
    if (rc) return rc;
    long long* S = (long long*)scr;
    BpBufs B;
    float* f5 = (float*)(S + o_f5);
    unsigned char* u2 = (unsigned char*)(S + o_u2);
    B.x = f5;
    B.y = f5 + nn;
    B.vx = f5 + 2 * nn;
    B.vy = f5 + 3 * nn;
    B.rr = f5 + 4 * nn;
    B.is_ast = u2;
    B.vis = u2 + nn;
    B.P = (const BpParams*)(S + o_par);
    B.counts = S + o_counts;
    B.scan_tmp = S + o_scan;
    B.cx = S + o_cx;
    B.cy = S + o_cy;
    B.k0 = (unsigned long long*)(S + o_k0);
    B.k1 = (unsigned long long*)(S + o_k1);
    B.v0 = (unsigned*)(S + o_v);
    B.v1 = B.v0 + nn;
    B.ai = (unsigned*)(S + o_ai);
    B.flags = S + o_flag;
    B.pos = S + o_pos;
    B.run_start = S + o_run;
    B.item_b0 = S + o_ib0;
    B.item_nb = S + o_inb;
    B.tile_st = S + o_tst;
    B.rec = (float4*)(S + o_rec);
    B.rec2 = (uint2*)(S + o_rec2);
    B.rowkey = (unsigned long long*)(S + o_rowkey);
    B.boxes = (ChunkBox*)(S + o_box);
    B.d_nh = (unsigned long long*)(S + o_nh);
    B.hits = (Hit*)(S + o_hits);

    // the graph of this size (captured on the first call of a size)
    sss_bp_graph* g = ctx->bp_graph;
    if (!g || g->n != nn || g->cap != capacity || g->base != scr) {
        sss_bp_graph_free(g);
        ctx->bp_graph = nullptr;
        g = new sss_bp_graph();
        cudaError_t e = cudaMallocHost((void**)&g->h_par, sizeof(BpParams));
        if (e == cudaSuccess) e = cudaMallocHost((void**)&g->h_cnt, 3 * sizeof(unsigned long long));
        if (e != cudaSuccess) {
            sss_bp_graph_free(g);
            return sss_cuda_err(ctx, e, "cudaMallocHost (broadphase graph)");
        }
        // capture on a private stream, so that the caller's stream never is in capture mode
        cudaStream_t cs;
        SSS_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        int prc = SSS_OK;
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync((void*)B.P, g->h_par, sizeof(BpParams), cudaMemcpyHostToDevice, cs);
            if (e == cudaSuccess) prc = enqueue_pipeline(ctx, B, nn, capacity, cs);
            if (e == cudaSuccess && prc == SSS_OK)
                e = cudaMemcpyAsync(g->h_cnt, B.d_nh, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, cs);
            if (e == cudaSuccess && prc == SSS_OK)
                e = cudaMemcpyAsync(g->h_cnt + 2, B.counts + tiles, sizeof(long long), cudaMemcpyDeviceToHost, cs);
            const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
            if (e == cudaSuccess) e = e2;
        }
        if (e == cudaSuccess && prc == SSS_OK) e = cudaGraphInstantiate(&g->exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (prc != SSS_OK || e != cudaSuccess) {
            sss_bp_graph_free(g);
            return prc != SSS_OK ? prc : sss_cuda_err(ctx, e, "broadphase graph capture");
        }
        g->n = nn;
        g->cap = capacity;
        g->base = scr;
        ctx->bp_graph = g;
    }
    g->h_par->lo = lo;
    g->h_par->hi_halo = hi + (float)halo;    // f32, as `self.hi + cp.float32(halo)`
    g->h_par->hi = hi;
    g->h_par->dtf = (float)dt_y;
    g->h_par->h = h;
    g->h_par->dt = dt_y;
    k_bp_stage<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(x, y, vx, vy, rr, is_ast, vis, nn, f5, u2);
    SSS_LAUNCH_CHECK(ctx, "k_bp_stage");
    SSS_CUDA_TRY(ctx, cudaGraphLaunch(g->exec, s));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    const unsigned long long nh = g->h_cnt[0], nc = g->h_cnt[1];
    const long long na = (long long)g->h_cnt[2];
    if (na < 2) return SSS_OK;                   // fewer than two alive asteroids: no candidates, no hits
    *n_cand = (int64_t)nc;
    *n_hits = (int64_t)nh;
    if ((long long)nh > capacity)
        return sss_set_err(ctx, SSS_ERR_CAPACITY, "hit buffer holds %lld, %llu hits found", (long long)capacity, nh);
    if (nh > 0)
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(out_hits, B.hits, (size_t)nh * sizeof(Hit), cudaMemcpyDeviceToDevice, s));
    return SSS_OK;
}

extern "C" int sss_broadphase_order(sss_ctx* ctx, int* hits, int64_t k, int64_t n, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (k < 0 || n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (k > 0 && !hits) return sss_set_err(ctx, SSS_ERR_ARG, "NULL hits");
    if (n >= ((int64_t)1 << 30)) return sss_set_err(ctx, SSS_ERR_ARG, "too many bodies for the packed hit key");
    if (k > (int64_t)INT32_MAX) return sss_set_err(ctx, SSS_ERR_ARG, "too many hits for the 32-bit sort index");
    if (k < 2) return SSS_OK;
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    int B = 1;
    while (((int64_t)1 << B) < n) ++B;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) & ~(size_t)255; return o; };
    const size_t o_k0 = take(8 * k), o_k1 = take(8 * k), o_v0 = take(4 * k), o_v1 = take(4 * k);
    const size_t o_tmp = take(12 * k), o_rs = take(8 * sss_dev::radix_scratch(k));
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* S = (char*)scr;
    unsigned long long* k0 = (unsigned long long*)(S + o_k0);
    unsigned long long* k1 = (unsigned long long*)(S + o_k1);
    unsigned* v0 = (unsigned*)(S + o_v0);
    unsigned* v1 = (unsigned*)(S + o_v1);
    Hit* tmp = (Hit*)(S + o_tmp);
    const unsigned nb = (unsigned)((k + 255) / 256);
    k_hit_keys<<<nb, 256, 0, s>>>((const Hit*)hits, k, B, k0, v0);
    SSS_LAUNCH_CHECK(ctx, "k_hit_keys");
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(k0, v0, k1, v1, k, (long long*)(S + o_rs), s, ctx->d_status, 3 + 2 * B));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(tmp, hits, 12 * (size_t)k, cudaMemcpyDeviceToDevice, s));
    k_hit_gather<<<nb, 256, 0, s>>>(tmp, v0, k, (Hit*)hits);
    SSS_LAUNCH_CHECK(ctx, "k_hit_gather");
    return SSS_OK;
}
