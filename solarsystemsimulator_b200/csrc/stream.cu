// The server's per-sample stream core on sm_100a (reference backend/server.py:
// build_frame :378-537 with _anzeige_koords :99-111, _lod_auswahl :629-684,
// _dichte_filter :686-747, _index_hash :117-131): display coordinates,
// culling by box and kill time, density LOD and u16 quantisation of one f32
// sample, with the reference's arithmetic (NumPy 2 promotion: f32 sample,
// Python floats cast to f32; f64 weights, bisection and rates).
//
// Per body the LOD needs only flags: the tier of a culled body (massive,
// asteroid of the system, injected asteroid), whether a density filter kept
// it. A density filter over a tier builds the 512 x 512 cell counts with
// integer atomics (order-free), finds the scale by the reference's 40-step
// bisection, whose f64 sums follow NumPy's pairwise summation over the
// 262,144 cells exactly (leaves of 128 cells with eight interleaved partial
// sums, then pairwise levels), turns it into per-cell rates and decides per
// body with the bilinear rate and the SplitMix64 hash of its index. The kept
// bodies are compacted in ascending order (the reference's np.sort of the
// concatenated tiers) and quantised in the same pass.
//
// The bisection uses that the sum is monotone in s (every term is, and
// rounded addition is monotone): its 40 decisions are those of the crossing
// point. Normally all of them come from the histogram of the cell counts
// (how many cells hold each count), with a certified error bound; where the
// bound cannot decide, rounds resolve 5 halvings each by summing the 31
// midpoints of the next 5 levels of the halving tree over all cells at once
// and reading the 5 decisions off them, each midpoint formed by the same
// arithmetic as the sequential halving.

#include "sss_internal.cuh"

#include <algorithm>

namespace {

constexpr int K = 512;                 // LOD cells per axis (server.py LOD_ZELLEN)
constexpr int K2 = K * K;
constexpr int LEAVES = K2 / 128;       // 2048 pairwise-sum leaves of 128 cells
constexpr double LOG33 = 3.4965075614664802;     // log(33) as the double the reference holds
constexpr float LOG33F = (float)LOG33;           // cast to f32 as NumPy casts the weak scalar

struct Box {
    float x0, y0, sx, sy;              // f32 of the Python floats x0, y0, spanx, spany
    float x1, y1;                      // f32 of x0 + spanx, y0 + spany (summed in f64)
};

// log(1 + x) for f32 x >= 0 with every operation rounded to f32, by the published reduction
// method of fdlibm's log1pf (Sun Microsystems, 1993): the f32 log1p of the C library that NumPy
// calls for float32 log1p where it dispatches no SIMD kernel. 1 + x = 2^k (1 + f) with
// sqrt(2)/2 <= 1 + f < sqrt(2) and a correction c for the rounding of 1 + x, s = f / (2 + f),
// log(1 + f) = f - (hfsq - s (hfsq + R(s^2))) with hfsq = f^2 / 2 and R a degree-7 minimax
// polynomial, k ln 2 in two parts; where k comes out 0 the correction is not applied.
__device__ __forceinline__ float log1p_f32(float x) {
    const int hx = __float_as_int(x);
    if (hx >= 0x7F800000 || hx < 0) return __fadd_rn(x, x);            // inf, nan (x < 0 never occurs)
    if (hx < 0x31000000)                                                // x < 2^-29
        return hx < 0x24800000 ? x : __fsub_rn(x, __fmul_rn(__fmul_rn(x, x), 0.5f));
    int k = 0, hu = 1;
    float f = x, c = 0.0f;
    if (hx >= 0x3ED413D7) {                                             // x >= 0.41422: reduce
        float u;
        if (hx < 0x5A000000) {
            u = __fadd_rn(1.0f, x);
            hu = __float_as_int(u);
            k = (hu >> 23) - 127;
            c = k > 0 ? __fsub_rn(1.0f, __fsub_rn(u, x)) : __fsub_rn(x, __fsub_rn(u, 1.0f));
            c = __fdiv_rn(c, u);
        } else {
            u = x;
            hu = __float_as_int(u);
            k = (hu >> 23) - 127;
        }
        hu &= 0x007FFFFF;
        if (hu < 0x3504F7) {
            u = __int_as_float(hu | 0x3F800000);
        } else {
            k += 1;
            u = __int_as_float(hu | 0x3F000000);
            hu = (0x00800000 - hu) >> 2;
        }
        f = __fsub_rn(u, 1.0f);
    }
    const float kf = (float)k;
    const float hfsq = __fmul_rn(__fmul_rn(0.5f, f), f);
    if (hu == 0) {                                                      // |f| < 2^-20
        if (f == 0.0f) return k == 0 ? 0.0f : __fadd_rn(__fmul_rn(kf, __int_as_float(0x3F317180)),
                                                        __fadd_rn(c, __fmul_rn(kf, __int_as_float(0x3717F7D1))));
        const float R = __fmul_rn(hfsq, __fsub_rn(1.0f, __fmul_rn(0.6666666666666666f, f)));
        if (k == 0) return __fsub_rn(f, R);
        return __fsub_rn(__fmul_rn(kf, __int_as_float(0x3F317180)),
                         __fsub_rn(__fsub_rn(R, __fadd_rn(__fmul_rn(kf, __int_as_float(0x3717F7D1)), c)), f));
    }
    const float s = __fdiv_rn(f, __fadd_rn(2.0f, f));
    const float z = __fmul_rn(s, s);
    float R = __int_as_float(0x3E178897);
    R = __fadd_rn(__int_as_float(0x3E1CD04F), __fmul_rn(z, R));
    R = __fadd_rn(__int_as_float(0x3E3A3325), __fmul_rn(z, R));
    R = __fadd_rn(__int_as_float(0x3E638E29), __fmul_rn(z, R));
    R = __fadd_rn(__int_as_float(0x3E924925), __fmul_rn(z, R));
    R = __fadd_rn(__int_as_float(0x3ECCCCCD), __fmul_rn(z, R));
    R = __fadd_rn(__int_as_float(0x3F2AAAAB), __fmul_rn(z, R));
    R = __fmul_rn(z, R);
    const float t = __fmul_rn(s, __fadd_rn(hfsq, R));
    if (k == 0) return __fsub_rn(f, __fsub_rn(hfsq, t));
    return __fsub_rn(__fmul_rn(kf, __int_as_float(0x3F317180)),
                     __fsub_rn(__fsub_rn(hfsq, __fadd_rn(t, __fadd_rn(__fmul_rn(kf, __int_as_float(0x3717F7D1)), c))),
                               f));
}

// Display scale of _anzeige_koords (server.py:99-111) for log zoom: log1p(r) / (log 33 * r) in
// f32, 0 at the origin.
__device__ __forceinline__ float log_zoom_scale(float px, float py) {
    const float r = sss_hypot_f32(px, py);
    return r > 1e-9f ? __fdiv_rn(log1p_f32(r), __fmul_rn(LOG33F, fmaxf(r, 1e-30f))) : 0.0f;
}

__global__ void k_disp(const float* __restrict__ x, const float* __restrict__ y, long long n, float* __restrict__ qx,
                       float* __restrict__ qy) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float sk = log_zoom_scale(x[i], y[i]);
    qx[i] = __fmul_rn(x[i], sk);
    qy[i] = __fmul_rn(y[i], sk);
}

__device__ __forceinline__ int cell_of(float q, float o, float s) {
    const int c = (int)__fmul_rn(__fdiv_rn(__fsub_rn(q, o), s), (float)K);
    return min(max(c, 0), K - 1);
}

__device__ __forceinline__ double index_hash(unsigned long long h) {
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 31;
    return (double)(h >> 11) / 9007199254740992.0;
}

__device__ __forceinline__ float frac_coord(float q, float o, float s) {
    const float f = __fsub_rn(__fmul_rn(__fdiv_rn(__fsub_rn(q, o), s), (float)K), 0.5f);
    return fminf(fmaxf(f, 0.0f), (float)(K - 1));
}

__device__ __forceinline__ unsigned short quant(float q, float o, float s) {
    const float v = __fmul_rn(__fdiv_rn(__fsub_rn(q, o), s), 65535.0f);
    return (unsigned short)fminf(fmaxf(v, 0.0f), 65535.0f);
}

__global__ void k_minmax(const float* __restrict__ qx, const float* __restrict__ qy, long long n,
                         float* __restrict__ out4) {
    __shared__ float s[4][256];
    float mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        mnx = fminf(mnx, qx[i]); mxx = fmaxf(mxx, qx[i]);
        mny = fminf(mny, qy[i]); mxy = fmaxf(mxy, qy[i]);
    }
    s[0][threadIdx.x] = mnx; s[1][threadIdx.x] = mxx; s[2][threadIdx.x] = mny; s[3][threadIdx.x] = mxy;
    __syncthreads();
    for (int w = 128; w; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s[0][threadIdx.x] = fminf(s[0][threadIdx.x], s[0][threadIdx.x + w]);
            s[1][threadIdx.x] = fmaxf(s[1][threadIdx.x], s[1][threadIdx.x + w]);
            s[2][threadIdx.x] = fminf(s[2][threadIdx.x], s[2][threadIdx.x + w]);
            s[3][threadIdx.x] = fmaxf(s[3][threadIdx.x], s[3][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out4[4 * blockIdx.x + 0] = s[0][0];
        out4[4 * blockIdx.x + 1] = s[1][0];
        out4[4 * blockIdx.x + 2] = s[2][0];
        out4[4 * blockIdx.x + 3] = s[3][0];
    }
}

size_t al(size_t b) { return (b + 255) / 256 * 256; }
unsigned nb(long long n) { return (unsigned)((n + 255) / 256); }

// ---------------------------------------------------------------- one sample
// The whole sample is one cooperative launch of SAMPLE_THREADS-thread blocks,
// all resident at once; its phases are separated by grid barriers:
//   cull      display coordinates, tier per body (keep = 0), tier counts of
//             the whole sample and of each block's range of bodies
//   (plan)    every block reads the tier counts and takes the reference's
//             branch of _lod_auswahl; the plan is uniform over the grid
//   filter    per thinned tier: cell counts (hist), the histogram of those
//             counts (values), the 40 halvings from it (block 0; rounds of
//             group sums over all cells for those it cannot decide), the
//             rate of every cell, keep decisions and kept counts per block
//   emit      each block places its range of bodies in ascending order
//             after those of the blocks before it
// A barrier wait polls at most BARRIER_POLLS times; when it runs out the
// block records SSS_ERR_TIMEOUT and every block returns at its next barrier.
constexpr int SAMPLE_THREADS = 512;
constexpr int SAMPLE_WARPS = SAMPLE_THREADS / 32;
constexpr unsigned BARRIER_POLLS = 1u << 21;        // about a second with the 32 ns back-off
constexpr int HIST_CHUNK = SAMPLE_THREADS * 4;      // bodies per shared-memory table fill
constexpr int HIST_SLOTS = 2 * HIST_CHUNK;          // 4096: the hash yields 12 bits
constexpr int EMIT_SUB = SAMPLE_THREADS * 8;        // bodies per block scan in the emit phase
constexpr int BISECT_D = 5;                         // halvings per round
constexpr int CAND = (1 << BISECT_D) - 1;           // 31 midpoints per round, lanes 0..30
constexpr int GROUP_LEAVES = SAMPLE_WARPS;          // 16 leaves of 128 cells per group (warp = leaf)
constexpr int GROUP_CELLS = GROUP_LEAVES * 128;
constexpr int GROUPS = LEAVES / GROUP_LEAVES;       // 128 groups
static_assert(HIST_SLOTS == 1 << 12, "12-bit hash");
static_assert(CAND < 32, "one lane per candidate");
static_assert(40 % BISECT_D == 0, "whole rounds of halvings");

struct Ctl {                                        // zeroed before every launch
    unsigned bar;                                   // grid barrier arrivals
    int err;
    unsigned long long tier_cnt[4];
    unsigned long long kept[2];
    long long total;
    int value_over[2];                              // per filter slot: more large distinct counts than vkey holds
    int fast_steps;                                 // halvings decided from the value histogram
    double lohi[2];                                 // the bisection interval after them
};

constexpr int VDIR = 4096;                          // cell counts below this: a table indexed by the count
constexpr int LSLOTS = 2048;                        // a block's larger distinct counts (open addressing)
constexpr int VALUE_SLOTS = 8192;                   // the grid's larger distinct counts (open addressing)
constexpr int VALUE_MAX = 4096;                     // at most this many distinct counts take the fast path
constexpr int SPRE_MAX = 1024;                      // fewer: their prefix sums are kept in shared memory

// the per-block record of blk: [1..3] bodies of tiers 1..3, [4 + slot] kept
// by the filter of that slot (a block of bodies: the contiguous range
// body_range gives it in the cull, keep and emit phases)
constexpr int BLK = 8;

struct SampleArgs {
    const float* x;
    const float* y;
    const double* kill_t;
    const unsigned char* is_ast;
    const unsigned char* injected;                  // may be NULL
    double t_cut;
    Box b;
    int log_zoom;
    long long n, budget;
    float* qx;                                      // display coordinates (log zoom), n
    float* qy;
    unsigned char* tier;                            // n
    unsigned char* keep;                            // n
    int* counts;                                    // 2 x K2 cell counts, one table per filter slot
    double* rate;                                   // K2 keep rates per cell
    double* part;                                   // 2 x CAND x GROUPS group sums
    long long* blk;                                 // BLK x gridDim.x: per block of bodies, its tier counts, kept counts
    unsigned* sel;
    unsigned short* ox;
    unsigned short* oy;
    Ctl* ctl;
    unsigned* vdir;                                 // 2 x VDIR: cells holding each count below VDIR
    int* vkey;                                      // 2 x VALUE_SLOTS: count value >= VDIR, -1 empty
    unsigned* vmul;                                 // 2 x VALUE_SLOTS: cells holding it
    double* vpre;                                   // 2 VALUE_MAX: prefix sums of the sorted values
};

// the count tables of one filter slot (each filter of a launch has its own,
// all cleared in the cull phase)
struct Tables {
    int* counts;
    unsigned* vdir;
    int* vkey;
    unsigned* vmul;
    int* over;
};

__device__ __forceinline__ Tables tables(const SampleArgs& a, int slot) {
    return Tables{a.counts + (size_t)slot * K2, a.vdir + slot * VDIR, a.vkey + slot * VALUE_SLOTS,
                  a.vmul + slot * VALUE_SLOTS, a.ctl->value_over + slot};
}

// bodies [c0, c1) of this block in the cull, keep and emit phases (c0 a
// multiple of 8)
__device__ __forceinline__ void body_range(long long n, long long& c0, long long& c1) {
    const long long chunk = ((n + gridDim.x - 1) / gridDim.x + 7) / 8 * 8;
    c0 = min((long long)blockIdx.x * chunk, n);
    c1 = min(c0 + chunk, n);
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// false: a wait ran out here or in another block (the caller returns)
__device__ __forceinline__ bool grid_barrier(Ctl* ctl, unsigned& epoch, int* s_bad,
                                             unsigned max_polls = BARRIER_POLLS) {
    ++epoch;
    __syncthreads();
    if (threadIdx.x == 0) {
        // release: the block's writes (ordered before this thread by the
        // block barrier) become visible with the arrival; acquire: the
        // other blocks' writes are visible once their arrivals are seen
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&ctl->bar) : "memory");
        const unsigned target = epoch * gridDim.x;
        int bad = 0;
        for (unsigned polls = 0; ld_acquire_u32(&ctl->bar) < target; ++polls) {
            if (polls >= max_polls || *(volatile int*)&ctl->err) {
                atomicExch(&ctl->err, SSS_ERR_TIMEOUT);
                bad = 1;
                break;
            }
            __nanosleep(32);
        }
        *s_bad = bad;
    }
    __syncthreads();
    return !*s_bad;
}

__device__ __forceinline__ long long block_sum_ll(long long v, long long* s_red) {
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = 0;
#pragma unroll
    for (int w = 0; w < SAMPLE_WARPS; ++w) t += s_red[w];
    return t;
}

// midpoint of heap node h (1-based) of the halving tree below [lo, hi]
__device__ __forceinline__ double node_mid(int h, double lo, double hi) {
    const int depth = 31 - __clz(h);
    for (int b = depth - 1; b >= 0; --b) {
        const double s = __dmul_rn(0.5, __dadd_rn(lo, hi));
        if ((h >> b) & 1) lo = s;
        else hi = s;
    }
    return __dmul_rn(0.5, __dadd_rn(lo, hi));
}

// weight of a cell: count ** 0.5 (a correctly rounded square root)
__device__ __forceinline__ double cell_weight(int c) { return c > 0 ? __dsqrt_rn((double)c) : 0.0; }

struct Smem {
    union {
        struct {                                    // hist phase
            int key[HIST_SLOTS];
            int val[HIST_SLOTS];
        } h;
        struct {                                    // values phase
            unsigned dir[VDIR];                     // cells per count below VDIR
            int lkey[LSLOTS];                       // larger counts
            unsigned lval[LSLOTS];
        } v;
        struct {                                    // bisection: one group's cells
            double c[GROUP_CELLS];
            double w[GROUP_CELLS];
        } g;
    } u;
    double leaf[GROUP_LEAVES][32];
    double tot[32];
    double dred[SAMPLE_WARPS];
    double dred2[SAMPLE_WARPS];
    long long red[SAMPLE_WARPS];
    int wcnt[SAMPLE_WARPS];
    int bad;
};

// Cell counts of the bodies whose tier is in mask: each block fills a
// shared-memory open-addressing table from HIST_CHUNK bodies (dense clouds
// put many bodies of a chunk into a few cells) and adds every distinct cell
// to the global counts once. The table has twice the chunk's slots, so a
// probe ends within HIST_SLOTS steps.
__device__ void phase_hist(const SampleArgs& a, const Tables& tb, const float* qx, const float* qy, int mask,
                           Smem& sm) {
    for (long long c0 = (long long)blockIdx.x * HIST_CHUNK; c0 < a.n; c0 += (long long)gridDim.x * HIST_CHUNK) {
        for (int j = threadIdx.x; j < HIST_SLOTS; j += SAMPLE_THREADS) {
            sm.u.h.key[j] = -1;
            sm.u.h.val[j] = 0;
        }
        __syncthreads();
        constexpr int R = HIST_CHUNK / SAMPLE_THREADS;
        int cells[R];                                            // -1: not in this filter's tiers
#pragma unroll
        for (int r = 0; r < R; ++r) {                           // all loads first: one latency for the chunk
            const long long i = c0 + (long long)r * SAMPLE_THREADS + threadIdx.x;
            const bool ok = i < a.n;
            const unsigned char t = ok ? __ldcg(a.tier + i) : 0;
            const float px = ok ? __ldcg(qx + i) : 0.0f, py = ok ? __ldcg(qy + i) : 0.0f;
            cells[r] = (mask >> t) & 1 ? cell_of(py, a.b.y0, a.b.sy) * K + cell_of(px, a.b.x0, a.b.sx) : -1;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int c = cells[r];
            if (c < 0) continue;
            unsigned h = ((unsigned)c * 2654435761u) >> 20;       // Fibonacci hash to 12 bits
            for (int probe = 0; probe < HIST_SLOTS; ++probe) {
                int k = *(volatile int*)(sm.u.h.key + h);
                if (k == -1) {
                    k = atomicCAS(sm.u.h.key + h, -1, c);
                    if (k == -1) k = c;                              // this lane took the slot
                }
                if (k == c) {
                    atomicAdd(sm.u.h.val + h, 1);
                    break;
                }
                h = (h + 1) & (HIST_SLOTS - 1);
            }
        }
        __syncthreads();
        for (int j = threadIdx.x; j < HIST_SLOTS; j += SAMPLE_THREADS)
            if (sm.u.h.key[j] >= 0) atomicAdd(tb.counts + sm.u.h.key[j], sm.u.h.val[j]);
        __syncthreads();
    }
}

// Group sums of the CAND midpoints below [lo, hi] for the groups of this
// block: warp = leaf of 128 cells (NumPy's pairwise leaf: eight interleaved
// partial sums, combined ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7))), lane =
// midpoint; then the 4 pairwise levels over the group's 16 leaves. A leaf of
// empty cells sums to +0 for every midpoint, as its terms min(0, s * 0) = +0
// do; in a leaf with occupied cells the +0 terms of its empty cells are added
// like the others (exactly).
__device__ void phase_group_sums(const Tables& tb, double lo, double hi, double* part, Smem& sm) {
    const int leaf = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int g = blockIdx.x; g < GROUPS; g += gridDim.x) {
        constexpr int PER_T = GROUP_CELLS / SAMPLE_THREADS;
        int cv[PER_T];
#pragma unroll
        for (int k = 0; k < PER_T; ++k) cv[k] = __ldcg(tb.counts + g * GROUP_CELLS + k * SAMPLE_THREADS + threadIdx.x);
#pragma unroll
        for (int k = 0; k < PER_T; ++k) {
            sm.u.g.c[k * SAMPLE_THREADS + threadIdx.x] = (double)cv[k];
            sm.u.g.w[k * SAMPLE_THREADS + threadIdx.x] = cell_weight(cv[k]);
        }
        __syncthreads();
        bool occ = false;
        for (int j = lane; j < 128; j += 32) occ |= sm.u.g.c[leaf * 128 + j] != 0.0;
        occ = __any_sync(0xffffffffu, occ);
        if (lane < CAND) {
            double sum = 0.0;
            if (occ) {
                const double s = node_mid(lane + 1, lo, hi);
                const double* c = sm.u.g.c + leaf * 128;
                const double* w = sm.u.g.w + leaf * 128;
                double r[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) r[j] = fmin(c[j], __dmul_rn(s, w[j]));
                for (int i = 8; i < 128; i += 8)
#pragma unroll
                    for (int j = 0; j < 8; ++j) r[j] = __dadd_rn(r[j], fmin(c[i + j], __dmul_rn(s, w[i + j])));
                sum = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                                __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
            }
            sm.leaf[leaf][lane] = sum;
        }
        __syncthreads();
        for (int m = GROUP_LEAVES / 2; m >= 1; m >>= 1) {
            double v = 0.0;
            if (leaf < m && lane < CAND) v = __dadd_rn(sm.leaf[2 * leaf][lane], sm.leaf[2 * leaf + 1][lane]);
            __syncthreads();
            if (leaf < m && lane < CAND) sm.leaf[leaf][lane] = v;
            __syncthreads();
        }
        if (threadIdx.x < CAND) part[threadIdx.x * GROUPS + g] = sm.leaf[0][threadIdx.x];
        __syncthreads();
    }
}

// the top 7 pairwise levels over the 128 group sums of every midpoint (a
// warp per midpoint: lane l adds groups 4l..4l+3 in two levels, then five
// shuffle levels pair lanes (l, l + d) for d = 1, 2, 4, 8, 16), then the
// BISECT_D decisions, taken alike by every block
static_assert(GROUPS == 4 * 32, "four group sums per lane");
__device__ void phase_walk(const double* part, double budget, double& lo, double& hi, int levels, Smem& sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < CAND; c += SAMPLE_WARPS) {
        const double2 p0 = __ldcg((const double2*)(part + c * GROUPS + 4 * lane));
        const double2 p1 = __ldcg((const double2*)(part + c * GROUPS + 4 * lane + 2));
        double v = __dadd_rn(__dadd_rn(p0.x, p0.y), __dadd_rn(p1.x, p1.y));
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, d);
            if ((lane & (2 * d - 1)) == 0) v = __dadd_rn(v, o);
        }
        if (lane == 0) sm.tot[c] = v;
    }
    __syncthreads();
    int node = 1;
    for (int d = 0; d < levels; ++d) {
        const double s = __dmul_rn(0.5, __dadd_rn(lo, hi));
        if (sm.tot[node - 1] > budget) {
            hi = s;
            node = 2 * node;
        } else {
            lo = s;
            node = 2 * node + 1;
        }
    }
}

__device__ __forceinline__ long long block_excl_scan_ll(long long v, Smem& sm, long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    __syncthreads();
    if (lane == 31) sm.red[warp] = inc;
    __syncthreads();
    long long before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < SAMPLE_WARPS; ++w) {
        const long long x = sm.red[w];
        before += w < warp ? x : 0;
        all += x;
    }
    *total = all;
    return before + inc - v;
}

// two exclusive block scans of doubles at once: shuffle scans in each warp,
// then the warp totals added in warp order; a thread's exclusive value is
// its inclusive one minus its own term
__device__ __forceinline__ void block_excl_scan_d2(double va, double vb, Smem& sm, double& ea, double& eb,
                                                   double& ta, double& tb) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double ia = va, ib = vb;
    for (int o = 1; o < 32; o <<= 1) {
        const double xa = __shfl_up_sync(0xffffffffu, ia, o), xb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o) {
            ia += xa;
            ib += xb;
        }
    }
    __syncthreads();
    if (lane == 31) {
        sm.dred[warp] = ia;
        sm.dred2[warp] = ib;
    }
    __syncthreads();
    double ba = 0.0, aa = 0.0, bb = 0.0, ab = 0.0;
#pragma unroll
    for (int w = 0; w < SAMPLE_WARPS; ++w) {
        const double xa = sm.dred[w], xb = sm.dred2[w];
        if (w < warp) {
            ba += xa;
            bb += xb;
        }
        aa += xa;
        ab += xb;
    }
    ta = aa;
    tb = ab;
    ea = ba + (ia - va);
    eb = bb + (ib - vb);
}

__device__ __forceinline__ void value_insert(const Tables& tb, int v, unsigned m) {
    unsigned h = ((unsigned)v * 2654435761u) >> 19;                  // Fibonacci hash to 13 bits
    for (int probe = 0; probe < VALUE_SLOTS; ++probe) {
        const int prev = atomicCAS(tb.vkey + h, -1, v);
        if (prev == -1 || prev == v) {
            atomicAdd(tb.vmul + h, m);
            return;
        }
        h = (h + 1) & (VALUE_SLOTS - 1);
    }
    atomicExch(tb.over, 1);
}
static_assert(VALUE_SLOTS == 1 << 13, "13-bit hash");

// The histogram of the nonzero cell counts (how many cells hold each count):
// each block takes a contiguous range of cells and merges them in shared
// memory, the counts below VDIR in a table indexed by the count and the
// larger ones in an open-addressing table, then adds them to the global
// tables (vdir, and vkey/vmul for the larger counts). A global table of
// larger counts that runs out of slots sets value_over (the bisection then
// takes the exact path).
__device__ void phase_values(const Tables& tb, Smem& sm) {
    for (int j = threadIdx.x; j < VDIR; j += SAMPLE_THREADS) sm.u.v.dir[j] = 0;
    for (int j = threadIdx.x; j < LSLOTS; j += SAMPLE_THREADS) {
        sm.u.v.lkey[j] = -1;
        sm.u.v.lval[j] = 0;
    }
    __syncthreads();
    const long long per = (K2 + gridDim.x - 1) / gridDim.x;
    const long long c0 = (long long)blockIdx.x * per, c1 = min(c0 + per, (long long)K2);
    for (long long c = c0 + threadIdx.x; c < c1; c += SAMPLE_THREADS) {
        const int v = __ldcg(tb.counts + c);
        if (v <= 0) continue;
        if (v < VDIR) {
            atomicAdd(sm.u.v.dir + v, 1u);
            continue;
        }
        unsigned h = ((unsigned)v * 2654435761u) >> 21;              // 11 bits
        bool done = false;
        for (int probe = 0; probe < LSLOTS; ++probe) {
            const int prev = atomicCAS(sm.u.v.lkey + h, -1, v);
            if (prev == -1 || prev == v) {
                atomicAdd(sm.u.v.lval + h, 1u);
                done = true;
                break;
            }
            h = (h + 1) & (LSLOTS - 1);
        }
        if (!done) value_insert(tb, v, 1u);                          // a full block table: straight to the global one
    }
    __syncthreads();
    for (int j = threadIdx.x; j < VDIR; j += SAMPLE_THREADS)
        if (sm.u.v.dir[j]) atomicAdd(tb.vdir + j, sm.u.v.dir[j]);
    for (int j = threadIdx.x; j < LSLOTS; j += SAMPLE_THREADS)
        if (sm.u.v.lkey[j] >= 0) value_insert(tb, sm.u.v.lkey[j], sm.u.v.lval[j]);
    __syncthreads();
}
static_assert(LSLOTS == 1 << 11, "11-bit hash");
static_assert(VDIR == 8 * SAMPLE_THREADS, "eight direct counts per thread");

// Ascending bitonic sort of n (a power of two) (value, cells) pairs in
// shared memory by the block. A stage of stride <= 32 pairs positions inside
// the 64 that one warp's 32 pairs cover (pair i of a stage: positions
// 2 i - (i mod stride) and that + stride), so between two such stages a
// warp synchronises only itself.
__device__ void block_bitonic(int* sv, int* sn, int n) {
    for (int size = 2; size <= n; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < n / 2; i += SAMPLE_THREADS) {
                const int l = 2 * i - (i & (stride - 1)), r = l + stride;
                const bool up = (l & size) == 0;
                const int vl = sv[l], vr = sv[r];
                if ((vl > vr) == up) {
                    const int nl = sn[l];
                    sv[l] = vr;
                    sv[r] = vl;
                    sn[l] = sn[r];
                    sn[r] = nl;
                }
            }
            const int next = stride > 1 ? stride >> 1 : size;      // the following stage's stride
            if (stride > 32 || next > 32) __syncthreads();
            else __syncwarp();
        }
    __syncthreads();
}

// The bisection from the count histogram (block 0). With the D distinct
// counts v_i sorted ascending, n_i the cells holding each, w_i = v_i ** 0.5
// and s the midpoint, the reference's sum over the cells of min(v, s w) is,
// up to rounding, F(s) = A_k + s (W - W_k), k the number of values with
// v_i <= s^2, A_k = sum_{i<k} n_i v_i (exact: integers below 2^53), W_k =
// sum_{i<k} n_i w_i, W = W_D. A halving is taken only where the decision
// F(s) > budget is certain: the reference's pairwise f64 sum differs from
// the exact sum of its terms by less than 30 ulp of it (leaves of 128 with
// 8 partial sums: 16 + 3 additions, 11 pairwise levels), the terms differ
// from those of F by less than 2 ulp of max(v, s w) (the classification
// at v = s^2 included), and the prefix sums here err by less than 30 ulp of
// W; so |f(s) - F(s)| < 1e-13 (F + s W + budget) with a wide margin. At the
// first step inside that margin the walk stops; the exact rounds finish it.
// The counts below VDIR come sorted from their direct table (thread t holds
// counts 8 t .. 8 t + 7); only the larger ones are sorted here.
__device__ void block_fast_bisection(const SampleArgs& a, const Tables& tb, double budget, Smem& sm) {
    int* sv = sm.u.h.key;                                            // sorted values (VALUE_MAX)
    int* sn = sm.u.h.val;                                            // their cell counts
    static_assert(HIST_SLOTS >= VALUE_MAX, "sort space");
    static_assert(2 * SPRE_MAX * sizeof(double) <= HIST_SLOTS * sizeof(int) && SPRE_MAX <= 2 * SAMPLE_THREADS,
                  "shared prefix sums fit the counts' space, two values per thread");
    constexpr int PER = VALUE_SLOTS / SAMPLE_THREADS;
    static_assert(PER % 4 == 0 && PER <= 32, "int4 loads of the large-count slots, one mask word");
    // the tables were filled by every block before the last grid barrier,
    // whose acquire orders those writes before these (L1-cached) loads
    const int* lkey = tb.vkey + threadIdx.x * PER;
    const int over = *tb.over;
    asm volatile("prefetch.global.L1 [%0];" ::"l"(tb.vmul + threadIdx.x * PER));  // read below for the occupied slots
    unsigned dn[8], lmask = 0;
    {
        const uint4 d0 = *(const uint4*)(tb.vdir + 8 * threadIdx.x);
        const uint4 d1 = *(const uint4*)(tb.vdir + 8 * threadIdx.x + 4);
        dn[0] = d0.x; dn[1] = d0.y; dn[2] = d0.z; dn[3] = d0.w;
        dn[4] = d1.x; dn[5] = d1.y; dn[6] = d1.z; dn[7] = d1.w;
    }
#pragma unroll
    for (int q = 0; q < PER; q += 4) {
        const int4 k4 = *(const int4*)(lkey + q);
        lmask |= (k4.x >= 0 ? 1u : 0u) << q | (k4.y >= 0 ? 2u : 0u) << q | (k4.z >= 0 ? 4u : 0u) << q |
                 (k4.w >= 0 ? 8u : 0u) << q;
    }
    int cs = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) cs += dn[q] != 0;
    const int cl = __popc(lmask);
    long long total = 0;                                             // (small << 32) + large, both < 2^14
    const long long off = block_excl_scan_ll(((long long)cs << 32) + cl, sm, &total);
    const int Ds = (int)(total >> 32), Dl = (int)(total & 0xffffffffLL);
    const int D = Ds + Dl;
    int Dlp = Dl > 0 ? 1 : 0;
    while (Dlp < Dl) Dlp <<= 1;
    if (over != 0 || D > VALUE_MAX || D < 1 || Ds + Dlp > HIST_SLOTS) {
        if (threadIdx.x == 0) {
            a.ctl->lohi[0] = 0.0;
            a.ctl->lohi[1] = budget;
            a.ctl->fast_steps = 0;
        }
        return;
    }
    {
        int w = (int)(off >> 32);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (dn[q]) {
                sv[w] = 8 * threadIdx.x + q;
                sn[w] = (int)dn[q];
                ++w;
            }
        w = Ds + (int)(off & 0xffffffffLL);
        for (unsigned m = lmask; m; m &= m - 1) {
            const int q = __ffs(m) - 1;
            sv[w] = lkey[q];
            sn[w] = (int)tb.vmul[threadIdx.x * PER + q];
            ++w;
        }
    }
    for (int i = Ds + Dl + threadIdx.x; i < Ds + Dlp; i += SAMPLE_THREADS) {
        sv[i] = INT_MAX;
        sn[i] = 0;
    }
    __syncthreads();
    if (Dl > 1 && Dl <= SAMPLE_THREADS) {
        // the larger counts (all >= VDIR, distinct): each of Dl threads
        // counts the smaller ones, then places its own
        int v = 0, c = 0, rank = 0;
        if ((int)threadIdx.x < Dl) {
            v = sv[Ds + threadIdx.x];
            c = sn[Ds + threadIdx.x];
            for (int j = 0; j < Dl; ++j) rank += sv[Ds + j] < v;
        }
        __syncthreads();
        if ((int)threadIdx.x < Dl) {
            sv[Ds + rank] = v;
            sn[Ds + rank] = c;
        }
        __syncthreads();
    } else if (Dl > 1) {
        block_bitonic(sv + Ds, sn + Ds, Dlp);
    }
    // prefix sums over chunks of consecutive values, then across the chunks.
    // With D < SPRE_MAX (at most 2 values per thread) they replace the cell
    // counts in shared memory (each thread keeps its own counts in
    // registers), else they go to global memory.
    const int ch = (D + SAMPLE_THREADS - 1) / SAMPLE_THREADS;
    const int i0 = threadIdx.x * ch, i1 = min(i0 + ch, D);
    const bool in_smem = D < SPRE_MAX;
    double* pre = in_smem ? (double*)sn : a.vpre;
    int n0 = 0, n1 = 0;
    double la = 0.0, lw = 0.0;
    for (int i = i0; i < i1; ++i) {
        const int c = sn[i];
        if (i == i0) n0 = c;
        else n1 = c;
        la += (double)c * (double)sv[i];
        lw += (double)c * cell_weight(sv[i]);
    }
    double tot_a, tot_w, ea, ew;
    block_excl_scan_d2(la, lw, sm, ea, ew, tot_a, tot_w);           // (its barriers end the reads of sn)
    for (int i = i0; i < i1; ++i) {
        const int c = !in_smem ? sn[i] : (i == i0 ? n0 : n1);
        pre[2 * i] = ea;
        pre[2 * i + 1] = ew;
        ea += (double)c * (double)sv[i];
        ew += (double)c * cell_weight(sv[i]);
    }
    if (threadIdx.x == 0) {
        pre[2 * D] = tot_a;
        pre[2 * D + 1] = tot_w;
    }
    __syncthreads();
    // warp 0. F at the breakpoints b_i = v_i ** 0.5 (where k = i + 1) grows
    // with i: a 32-way search finds the piece on which F crosses the budget,
    // and that piece's line gives an estimate s_est of the crossing. The
    // reference's sum grows with s (each term min(c, s w) does, and so does a
    // rounded sum), so its halvings go up exactly where the midpoint lies
    // above its crossing: the 40 halvings the estimate predicts are checked
    // at once (step j on lane j and lane j - 32), each taken when F at its
    // midpoint certainly lies on the predicted side of the budget, up to the
    // first that is not. Where that leaves steps, rounds of BISECT_D
    // halvings go on from there, lane c evaluating the midpoint of node c + 1
    // of the halving tree below (lo, hi) (node_mid: the same arithmetic as
    // the sequential halving), the certain decisions in two ballots, up to
    // the first uncertain node. k(s) grows with s, so inside [lo, hi] it
    // lies between the k of the nodes that set lo and hi.
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const double W = tot_w;
        int bl = -1, bh = D;                                         // F(b_bl) <= budget < F(b_bh), virtual ends
        while (bh - bl > 1) {
            const int step = (bh - bl + 31) / 32;
            const int i = bl + (lane + 1) * step;
            bool le = false;
            if (i < bh) le = pre[2 * i + 2] + cell_weight(sv[i]) * (W - pre[2 * i + 3]) <= budget;
            const int c = __popc(__ballot_sync(0xffffffffu, le));
            bh = min(bh, bl + (c + 1) * step);
            bl += c * step;
        }
        const double den = W - pre[2 * (bl + 1) + 1];
        const double s_est = den > 0.0 ? (budget - pre[2 * (bl + 1)]) / den : budget;
        double lo = 0.0, hi = budget, s0 = 0.0, s1 = 0.0, lo0 = 0.0, hi0 = 0.0, lo1 = 0.0, hi1 = 0.0;
        bool p0 = false, p1 = false;
        for (int j = 0; j < 40; ++j) {                               // lane j (and j - 32) keeps step j and the interval after it
            const double s = __dmul_rn(0.5, __dadd_rn(lo, hi));
            const bool up = s > s_est;
            if (up) hi = s;
            else lo = s;
            if (j == lane) {
                s0 = s;
                p0 = up;
                lo0 = lo;
                hi0 = hi;
            }
            if (j == lane + 32) {
                s1 = s;
                p1 = up;
                lo1 = lo;
                hi1 = hi;
            }
        }
        auto certain = [&](double s, bool up) {
            const double s2 = s * s;
            int l = 0, r = D;                                        // k = #values <= s^2
            while (l < r) {
                const int m = (l + r) >> 1;
                if ((double)sv[m] <= s2) l = m + 1;
                else r = m;
            }
            const double F = pre[2 * l] + s * (W - pre[2 * l + 1]);
            const double margin = 1e-13 * (F + s * W + budget);
            return up ? F > budget + margin : F < budget - margin;
        };
        const unsigned ok0 = __ballot_sync(0xffffffffu, certain(s0, p0));
        const unsigned ok1 = __ballot_sync(0xffffffffu, lane >= 8 || certain(s1, p1));
        const unsigned long long bad = (unsigned long long)~ok0 | ((unsigned long long)(~ok1 & 0xffu) << 32);
        int steps = bad ? __ffsll((long long)bad) - 1 : 40;
        if (steps == 0) {
            lo = 0.0;
            hi = budget;
        } else {                                                     // the interval after step steps - 1
            const int j = steps - 1;
            lo = __shfl_sync(0xffffffffu, j < 32 ? lo0 : lo1, j & 31);
            hi = __shfl_sync(0xffffffffu, j < 32 ? hi0 : hi1, j & 31);
        }
        int klo = 0, khi = D;
        bool stop = false;
        while (steps < 40 && !stop) {
            int k = 0;
            bool up = false, down = false;
            if (lane < CAND) {
                const double s = node_mid(lane + 1, lo, hi);
                const double s2 = s * s;
                int l = klo, r = khi;                                // k = #values <= s^2
                while (l < r) {
                    const int m = (l + r) >> 1;
                    if ((double)sv[m] <= s2) l = m + 1;
                    else r = m;
                }
                k = l;
                const double F = pre[2 * l] + s * (W - pre[2 * l + 1]);
                const double margin = 1e-13 * (F + s * W + budget);
                up = F > budget + margin;
                down = F < budget - margin;
            }
            const unsigned b_up = __ballot_sync(0xffffffffu, up), b_down = __ballot_sync(0xffffffffu, down);
            const int levels = min(BISECT_D, 40 - steps);
            int node = 1, n_lo = 0, n_hi = 0;
            for (int d = 0; d < levels; ++d) {
                const double s = __dmul_rn(0.5, __dadd_rn(lo, hi));
                if ((b_up >> (node - 1)) & 1) {
                    hi = s;
                    n_hi = node;
                    node = 2 * node;
                } else if ((b_down >> (node - 1)) & 1) {
                    lo = s;
                    n_lo = node;
                    node = 2 * node + 1;
                } else {
                    stop = true;
                    break;
                }
                ++steps;
            }
            const int k_lo = __shfl_sync(0xffffffffu, k, max(n_lo - 1, 0));
            const int k_hi = __shfl_sync(0xffffffffu, k, max(n_hi - 1, 0));
            if (n_lo) klo = k_lo;
            if (n_hi) khi = k_hi;
        }
        if (lane == 0) {
            a.ctl->lohi[0] = lo;
            a.ctl->lohi[1] = hi;
            a.ctl->fast_steps = steps;
        }
    }
}

// The reference's _dichte_filter over the tiers in mask with `budget`
// points (size > budget); keep[i] = 1 for the kept bodies, their number in
// ctl->kept[slot] and, per block of bodies, in its record. Returns false
// when a barrier gave up.
__device__ bool filter(const SampleArgs& a, const float* qx, const float* qy, int mask, long long budget, int slot,
                       unsigned& epoch, Smem& sm) {
    const Tables tb = tables(a, slot);
    phase_hist(a, tb, qx, qy, mask, sm);
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    phase_values(tb, sm);
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    if (blockIdx.x == 0) block_fast_bisection(a, tb, (double)budget, sm);
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    // every thread reads the control words after a barrier: L1-cached loads,
    // so that one request per SM reaches their L2 line
    double lo = __ldca(&a.ctl->lohi[0]), hi = __ldca(&a.ctl->lohi[1]);
    // the halvings the histogram could not decide (normally none): exact rounds
    int left = 40 - __ldca(&a.ctl->fast_steps);
    for (int round = 0; left > 0; ++round) {
        double* part = a.part + (round & 1) * CAND * GROUPS;
        phase_group_sums(tb, lo, hi, part, sm);
        if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
        const int levels = min(BISECT_D, left);
        phase_walk(part, (double)budget, lo, hi, levels, sm);
        left -= levels;
    }
    const long long T = (long long)gridDim.x * SAMPLE_THREADS;
    const long long gt = (long long)blockIdx.x * SAMPLE_THREADS + threadIdx.x;
    // the keep rate of every cell: min(k, lo k ** 0.5) / k, 0 for an empty cell
    for (long long c = gt; c < K2; c += T) {
        const int k = __ldcg(tb.counts + c);
        a.rate[c] = k > 0 ? __ddiv_rn(fmin((double)k, __dmul_rn(lo, cell_weight(k))), (double)k) : 0.0;
    }
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    const unsigned char* __restrict__ tier = a.tier;
    unsigned char* __restrict__ keep = a.keep;
    const double* __restrict__ rate = a.rate;
    long long c0, c1;
    body_range(a.n, c0, c1);
    long long kept = 0;
    // two bodies per thread and pass, in three stages (loads, rate gathers,
    // decisions) so that both bodies' gathers are in flight together. A body
    // reads the rates of cells (iy, ix), (iy, ix1), (iy1, ix), (iy1, ix1)
    // for its bilinear rate. The gathers are plain (L1-cached) loads: a dense
    // cloud puts many bodies into the same few cells, and L2-only loads of
    // those rates queue at their L2 slices. The rates were written by other
    // blocks before the last grid barrier, whose acquire orders them before
    // these loads.
    for (long long i0 = c0 + threadIdx.x; i0 < c1; i0 += 2 * SAMPLE_THREADS) {
        bool in[2];
        float fx[2], fy[2];
        int ix[2], iy[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const long long i = i0 + u * SAMPLE_THREADS;
            const bool ok = i < c1;
            const unsigned char t = ok ? __ldcg(tier + i) : 0;
            const float px = ok ? __ldcg(qx + i) : 0.0f, py = ok ? __ldcg(qy + i) : 0.0f;
            in[u] = (mask >> t) & 1;
            fx[u] = frac_coord(px, a.b.x0, a.b.sx);
            fy[u] = frac_coord(py, a.b.y0, a.b.sy);
            ix[u] = (int)floorf(fx[u]);
            iy[u] = (int)floorf(fy[u]);
        }
        double r[2][4];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int x1 = min(ix[u] + 1, K - 1), y1 = min(iy[u] + 1, K - 1);
            const int cells[4] = {iy[u] * K + ix[u], iy[u] * K + x1, y1 * K + ix[u], y1 * K + x1};
#pragma unroll
            for (int q = 0; q < 4; ++q) r[u][q] = in[u] ? rate[cells[q]] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const long long i = i0 + u * SAMPLE_THREADS;
            const double tx = __dsub_rn((double)fx[u], (double)ix[u]), ty = __dsub_rn((double)fy[u], (double)iy[u]);
            const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
            double rp = __dmul_rn(__dmul_rn(r[u][0], ux), uy);
            rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(r[u][1], tx), uy));
            rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(r[u][2], ux), ty));
            rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(r[u][3], tx), ty));
            if (in[u] && index_hash((unsigned long long)i) < rp) {
                keep[i] = 1;
                ++kept;
            }
        }
    }
    kept = block_sum_ll(kept, sm.red);
    if (threadIdx.x == 0) {
        a.blk[(size_t)blockIdx.x * BLK + 4 + slot] = kept;
        if (kept) atomicAdd(a.ctl->kept + slot, (unsigned long long)kept);
    }
    return grid_barrier(a.ctl, epoch, &sm.bad);
}

__global__ void __launch_bounds__(SAMPLE_THREADS) k_sample(SampleArgs a) {
    __shared__ Smem sm;
    unsigned epoch = 0;
    const long long T = (long long)gridDim.x * SAMPLE_THREADS;
    const long long gt = (long long)blockIdx.x * SAMPLE_THREADS + threadIdx.x;
    const float* qx = a.log_zoom ? a.qx : a.x;
    const float* qy = a.log_zoom ? a.qy : a.y;
    // ---- cull (and clear both filter slots' count tables)
    long long n1 = 0, n2 = 0, n3 = 0;
    for (long long c = gt; c < 2 * K2; c += T) a.counts[c] = 0;
    for (long long c = gt; c < 2 * VALUE_SLOTS; c += T) {
        a.vkey[c] = -1;
        a.vmul[c] = 0;
    }
    for (long long c = gt; c < 2 * VDIR; c += T) a.vdir[c] = 0;
    long long c0, c1;
    body_range(a.n, c0, c1);
    for (long long i0 = c0 + threadIdx.x; i0 < c1; i0 += 4 * SAMPLE_THREADS) {
        float bx[4], by[4];
        double kt[4];
        unsigned char ast[4], inj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {                           // all loads first: one latency per pass
            const long long i = i0 + u * SAMPLE_THREADS;
            const bool ok = i < c1;
            bx[u] = ok ? a.x[i] : 0.0f;
            by[u] = ok ? a.y[i] : 0.0f;
            kt[u] = ok ? a.kill_t[i] : 0.0;
            ast[u] = ok ? a.is_ast[i] : 0;
            inj[u] = ok && a.injected ? a.injected[i] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long i = i0 + u * SAMPLE_THREADS;
            if (i >= c1) break;
            float px = bx[u], py = by[u];
            if (a.log_zoom) {
                const float sk = log_zoom_scale(px, py);
                px = __fmul_rn(px, sk);
                py = __fmul_rn(py, sk);
                a.qx[i] = px;
                a.qy[i] = py;
            }
            unsigned char t = 0;
            if ((kt[u] > a.t_cut) & (px >= a.b.x0) & (px <= a.b.x1) & (py >= a.b.y0) & (py <= a.b.y1))
                t = !ast[u] ? 1 : (inj[u] ? 3 : 2);
            a.tier[i] = t;
            a.keep[i] = 0;
            n1 += t == 1;
            n2 += t == 2;
            n3 += t == 3;
        }
    }
    n1 = block_sum_ll(n1, sm.red);
    n2 = block_sum_ll(n2, sm.red);
    n3 = block_sum_ll(n3, sm.red);
    if (threadIdx.x == 0) {
        if (n1) atomicAdd(a.ctl->tier_cnt + 1, (unsigned long long)n1);
        if (n2) atomicAdd(a.ctl->tier_cnt + 2, (unsigned long long)n2);
        if (n3) atomicAdd(a.ctl->tier_cnt + 3, (unsigned long long)n3);
        long long* rec = a.blk + (size_t)blockIdx.x * BLK;
        rec[1] = n1;
        rec[2] = n2;
        rec[3] = n3;
        rec[4] = 0;
        rec[5] = 0;
    }
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return;
    // ---- plan (the reference's _lod_auswahl), identical in every block
    // (every thread reads the counts: L1-cached loads, one L2 request per SM)
    const long long mm = (long long)__ldca(a.ctl->tier_cnt + 1), ma = (long long)__ldca(a.ctl->tier_cnt + 2),
                    mi = (long long)__ldca(a.ctl->tier_cnt + 3);
    const long long m = mm + ma + mi;
    const int T_ALL = (1 << 1) | (1 << 2) | (1 << 3), T_MASS = 1 << 1, T_AST = (1 << 2) | (1 << 3);
    int all_mask = 0;
    if (m <= a.budget) {
        all_mask = T_ALL;
    } else {
        long long rest = a.budget - mm;
        if (rest <= 0) {
            if (mm > 200 && m > mm) {
                // many massive bodies (a self-gravity cloud): they get half the budget, thinned
                const long long m_budget = max(1LL, (long long)((double)a.budget * 0.5));
                long long kept = mm;
                if (mm <= m_budget) {
                    all_mask |= T_MASS;
                } else {
                    if (!filter(a, qx, qy, T_MASS, m_budget, 0, epoch, sm)) return;
                    kept = (long long)__ldca(a.ctl->kept + 0);
                }
                rest = a.budget - kept;
                if (rest > 0 && ma + mi > 0) {
                    if (ma + mi <= rest) all_mask |= T_AST;
                    else if (!filter(a, qx, qy, T_AST, rest, 1, epoch, sm)) return;
                }
            } else {
                all_mask = T_MASS;
            }
        } else {
            all_mask = T_MASS;
            const long long sizes[2] = {ma, mi};
            const int masks[2] = {1 << 2, 1 << 3};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (rest <= 0 || sizes[q] == 0) continue;
                long long kept = sizes[q];
                if (sizes[q] <= rest) {
                    all_mask |= masks[q];
                } else {
                    if (!filter(a, qx, qy, masks[q], rest, q, epoch, sm)) return;
                    kept = (long long)__ldca(a.ctl->kept + q);
                }
                rest -= kept;
            }
        }
    }
    // ---- emit: block b places its bodies [c0, c1) after those of blocks
    // 0 .. b - 1. A block emits its kept bodies and its bodies of the tiers
    // in all_mask (never a filtered tier): its record holds both numbers.
    long long before = 0;
    for (int j = threadIdx.x; j < (int)blockIdx.x; j += SAMPLE_THREADS) {
        const long long* rec = a.blk + (size_t)j * BLK;
        long long e = __ldca(rec + 4) + __ldca(rec + 5);            // (read by every later block: L1-cached)
#pragma unroll
        for (int t = 1; t <= 3; ++t)
            if ((all_mask >> t) & 1) e += __ldca(rec + t);
        before += e;
    }
    long long off = block_sum_ll(before, sm.red);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // 8 consecutive bodies per thread: flags in one 8-byte load each, the
    // coordinates in float4 loads where both arrays are 16-byte aligned (the
    // ranges start at multiples of 8)
    const bool vec = ((reinterpret_cast<unsigned long long>(qx) | reinterpret_cast<unsigned long long>(qy)) & 15) == 0;
    for (long long s0 = c0; s0 < c1; s0 += EMIT_SUB) {
        const long long i0 = s0 + (long long)threadIdx.x * 8;
        unsigned bits = 0, oq[8];                                // oq: the quantised (x, y) of each body
        auto put = [&](int j, unsigned kp, unsigned t, float px, float py) {
            if (kp | ((all_mask >> t) & 1)) bits |= 1u << j;
            oq[j] = (unsigned)quant(px, a.b.x0, a.b.sx) | (unsigned)quant(py, a.b.y0, a.b.sy) << 16;
        };
        if (i0 + 7 < c1) {                                      // all loads first: one latency per sub-range
            const uint2 k8 = __ldcg((const uint2*)(a.keep + i0)), t8 = __ldcg((const uint2*)(a.tier + i0));
            float xs[8], ys[8];
            if (vec) {
                const float4 x0 = __ldcg((const float4*)(qx + i0)), x1 = __ldcg((const float4*)(qx + i0 + 4));
                const float4 y0 = __ldcg((const float4*)(qy + i0)), y1 = __ldcg((const float4*)(qy + i0 + 4));
                xs[0] = x0.x; xs[1] = x0.y; xs[2] = x0.z; xs[3] = x0.w;
                xs[4] = x1.x; xs[5] = x1.y; xs[6] = x1.z; xs[7] = x1.w;
                ys[0] = y0.x; ys[1] = y0.y; ys[2] = y0.z; ys[3] = y0.w;
                ys[4] = y1.x; ys[5] = y1.y; ys[6] = y1.z; ys[7] = y1.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    xs[j] = __ldcg(qx + i0 + j);
                    ys[j] = __ldcg(qy + i0 + j);
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const unsigned kw = j < 4 ? k8.x : k8.y, tw = j < 4 ? t8.x : t8.y, sh = 8 * (j & 3);
                put(j, (kw >> sh) & 0xffu, (tw >> sh) & 0xffu, xs[j], ys[j]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const long long i = i0 + j;
                oq[j] = 0;
                if (i < c1) put(j, __ldcg(a.keep + i), __ldcg(a.tier + i), __ldcg(qx + i), __ldcg(qy + i));
            }
        }
        const int c = __popc(bits);
        int inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) sm.wcnt[warp] = inc;
        __syncthreads();
        int wb = 0, all = 0;
#pragma unroll
        for (int w = 0; w < SAMPLE_WARPS; ++w) {
            const int v = sm.wcnt[w];
            wb += w < warp ? v : 0;
            all += v;
        }
        long long q = off + wb + inc - c;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (!((bits >> j) & 1)) continue;
            const long long i = i0 + j;
            a.sel[q] = (unsigned)i;
            a.ox[q] = (unsigned short)(oq[j] & 0xffffu);
            a.oy[q] = (unsigned short)(oq[j] >> 16);
            ++q;
        }
        off += all;
        __syncthreads();                            // wcnt is rewritten by the next sub-range
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) a.ctl->total = off;
}

struct Work {
    float *qx, *qy;
    unsigned char *tier, *keep;
    int* counts;
    double *rate, *part;
    unsigned* vdir;
    int* vkey;
    unsigned* vmul;
    double* vpre;
    long long* blk;
    Ctl* ctl;
};

// scratch of a sample (reused by the samples of a batch, which run in
// stream order) and n_ctl control blocks (one per sample of a batch)
int make_work(sss_ctx* ctx, long long n, int grid, int n_ctl, Work* W) {
    size_t off = 0;
    const size_t o_qx = off; off += al((size_t)n * 4);
    const size_t o_qy = off; off += al((size_t)n * 4);
    const size_t o_tier = off; off += al((size_t)n);
    const size_t o_keep = off; off += al((size_t)n);
    const size_t o_cnts = off; off += al((size_t)2 * K2 * 4);
    const size_t o_rate = off; off += al((size_t)K2 * 8);
    const size_t o_part = off; off += al((size_t)2 * CAND * GROUPS * 8);
    const size_t o_vdir = off; off += al((size_t)2 * VDIR * 4);
    const size_t o_vkey = off; off += al((size_t)2 * VALUE_SLOTS * 4);
    const size_t o_vmul = off; off += al((size_t)2 * VALUE_SLOTS * 4);
    const size_t o_vpre = off; off += al((size_t)2 * (VALUE_MAX + 1) * 8);
    const size_t o_blk = off; off += al((size_t)grid * BLK * 8);
    const size_t o_ctl = off; off += al(sizeof(Ctl) * (size_t)n_ctl);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* p = (char*)scr;
    W->qx = (float*)(p + o_qx);
    W->qy = (float*)(p + o_qy);
    W->tier = (unsigned char*)(p + o_tier);
    W->keep = (unsigned char*)(p + o_keep);
    W->counts = (int*)(p + o_cnts);
    W->rate = (double*)(p + o_rate);
    W->part = (double*)(p + o_part);
    W->vdir = (unsigned*)(p + o_vdir);
    W->vkey = (int*)(p + o_vkey);
    W->vmul = (unsigned*)(p + o_vmul);
    W->vpre = (double*)(p + o_vpre);
    W->blk = (long long*)(p + o_blk);
    W->ctl = (Ctl*)(p + o_ctl);
    return SSS_OK;
}

// blocks of one cooperative k_sample launch: every SM's resident blocks, at most 2 per SM
int sample_grid(sss_ctx* ctx, int* grid) {
    static int per_sm_of[64];                       // per device ordinal, 0 = not queried yet
    const int dev = ctx->device;
    int per_sm = dev >= 0 && dev < 64 ? per_sm_of[dev] : 0;
    if (per_sm == 0) {
        SSS_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sample, SAMPLE_THREADS, 0));
        if (per_sm < 1) return sss_set_err(ctx, SSS_ERR_CUDA, "k_sample: no resident block per SM");
        if (dev >= 0 && dev < 64) per_sm_of[dev] = per_sm;
    }
    *grid = ctx->num_sms * std::min(per_sm, 2);
    return SSS_OK;
}

}  // namespace

extern "C" int sss_stream_display(sss_ctx* ctx, int64_t n, const float* x, const float* y, float* qx, float* qy,
                                  void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (n < 0 || (n > 0 && (!x || !y || !qx || !qy)))
        return sss_set_err(ctx, SSS_ERR_ARG, "display: negative size or NULL buffer");
    if (n == 0) return SSS_OK;
    k_disp<<<nb(n), 256, 0, (cudaStream_t)stream>>>(x, y, n, qx, qy);
    SSS_LAUNCH_CHECK(ctx, "k_disp");
    return SSS_OK;
}

extern "C" int sss_stream_minmax(sss_ctx* ctx, int64_t n, const float* x, const float* y, int log_zoom, float* out4,
                                 void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (n < 1 || !x || !y || !out4) return sss_set_err(ctx, SSS_ERR_ARG, "minmax: empty or NULL input");
    cudaStream_t st = (cudaStream_t)stream;
    Work W;
    int rc = make_work(ctx, n, 1, 1, &W);
    if (rc) return rc;
    const float* qx = x;
    const float* qy = y;
    if (log_zoom) {
        k_disp<<<nb(n), 256, 0, st>>>(x, y, n, W.qx, W.qy);
        SSS_LAUNCH_CHECK(ctx, "k_disp");
        qx = W.qx;
        qy = W.qy;
    }
    const int blocks = (int)std::min<long long>(nb(n), 256);
    float* part = (float*)W.rate;                // 4 floats per block
    k_minmax<<<blocks, 256, 0, st>>>(qx, qy, n, part);
    SSS_LAUNCH_CHECK(ctx, "k_minmax");
    float h[4 * 256];
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(h, part, sizeof(float) * 4 * blocks, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    float r[4] = {h[0], h[1], h[2], h[3]};
    for (int bkt = 1; bkt < blocks; ++bkt) {
        r[0] = std::min(r[0], h[4 * bkt]);
        r[1] = std::max(r[1], h[4 * bkt + 1]);
        r[2] = std::min(r[2], h[4 * bkt + 2]);
        r[3] = std::max(r[3], h[4 * bkt + 3]);
    }
    for (int c = 0; c < 4; ++c) out4[c] = r[c];
    return SSS_OK;
}

namespace {

// k samples of the same bodies, one cooperative launch each in stream
// order, one readback of the k counts at the end
int sample_batch(sss_ctx* ctx, int64_t n, int k, const float* const* x, const float* const* y,
                 const double* kill_t, const double* t_cut, const unsigned char* is_ast,
                 const unsigned char* injected, const double* box, int log_zoom, int64_t budget, unsigned* sel,
                 uint16_t* qx_out, uint16_t* qy_out, int64_t* n_sel, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!n_sel || !box || (k > 0 && (!x || !y || !t_cut))) return sss_set_err(ctx, SSS_ERR_ARG, "NULL host array");
    if (k < 0 || k > 4096) return sss_set_err(ctx, SSS_ERR_ARG, "batch of 0..4096 samples");
    for (int i = 0; i < k; ++i) n_sel[i] = 0;
    if (n < 0 || budget < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n == 0 || k == 0) return SSS_OK;
    if (n > 0xFFFFFFFFLL) return sss_set_err(ctx, SSS_ERR_ARG, "more than 2^32 bodies (u32 indices)");
    if (!kill_t || !is_ast || !sel || !qx_out || !qy_out) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    for (int i = 0; i < k; ++i)
        if (!x[i] || !y[i]) return sss_set_err(ctx, SSS_ERR_ARG, "NULL sample %d", i);
    cudaStream_t st = (cudaStream_t)stream;
    int grid = 0;
    int rc = sample_grid(ctx, &grid);
    if (rc) return rc;
    Work W;
    rc = make_work(ctx, n, grid, k, &W);
    if (rc) return rc;
    SampleArgs a;
    a.kill_t = kill_t;
    a.is_ast = is_ast;
    a.injected = injected;
    a.b.x0 = (float)box[0];
    a.b.y0 = (float)box[1];
    a.b.sx = (float)box[2];
    a.b.sy = (float)box[3];
    a.b.x1 = (float)(box[0] + box[2]);
    a.b.y1 = (float)(box[1] + box[3]);
    a.log_zoom = log_zoom ? 1 : 0;
    a.n = n;
    a.budget = budget;
    a.qx = W.qx;
    a.qy = W.qy;
    a.tier = W.tier;
    a.keep = W.keep;
    a.counts = W.counts;
    a.rate = W.rate;
    a.part = W.part;
    a.blk = W.blk;
    a.vdir = W.vdir;
    a.vkey = W.vkey;
    a.vmul = W.vmul;
    a.vpre = W.vpre;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(W.ctl, 0, sizeof(Ctl) * (size_t)k, st));
    for (int i = 0; i < k; ++i) {
        a.x = x[i];
        a.y = y[i];
        a.t_cut = t_cut[i];
        a.sel = sel + (size_t)i * n;
        a.ox = qx_out + (size_t)i * n;
        a.oy = qy_out + (size_t)i * n;
        a.ctl = W.ctl + i;
        void* params[] = {&a};
        SSS_CUDA_TRY(ctx, cudaLaunchCooperativeKernel((const void*)k_sample, dim3(grid), dim3(SAMPLE_THREADS), params,
                                                      0, st));
    }
    Ctl hbuf[16];
    Ctl* h = k <= 16 ? hbuf : new Ctl[k];
    cudaError_t e = cudaMemcpyAsync(h, W.ctl, sizeof(Ctl) * (size_t)k, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    int bad = -1;
    if (e == cudaSuccess)
        for (int i = 0; i < k; ++i) {
            if (h[i].err && bad < 0) bad = i;
            n_sel[i] = h[i].total;
        }
    if (h != hbuf) delete[] h;
    if (e != cudaSuccess) return sss_cuda_err(ctx, e, "stream sample readback");
    if (bad >= 0) {
        for (int i = 0; i < k; ++i) n_sel[i] = 0;
        return sss_set_err(ctx, SSS_ERR_TIMEOUT, "k_sample (sample %d): a grid barrier wait ran out", bad);
    }
    return SSS_OK;
}

}  // namespace

extern "C" int sss_stream_sample(sss_ctx* ctx, int64_t n, const float* x, const float* y, const double* kill_t,
                                 double t_cut, const unsigned char* is_ast, const unsigned char* injected,
                                 const double* box, int log_zoom, int64_t budget, unsigned* sel, uint16_t* qx_out,
                                 uint16_t* qy_out, int64_t* n_sel, void* stream) {
    return sample_batch(ctx, n, 1, &x, &y, kill_t, &t_cut, is_ast, injected, box, log_zoom, budget, sel, qx_out,
                        qy_out, n_sel, stream);
}

extern "C" int sss_stream_sample_batch(sss_ctx* ctx, int64_t n, int k, const float* const* x, const float* const* y,
                                       const double* kill_t, const double* t_cut, const unsigned char* is_ast,
                                       const unsigned char* injected, const double* box, int log_zoom,
                                       int64_t budget, unsigned* sel, uint16_t* qx_out, uint16_t* qy_out,
                                       int64_t* n_sel, void* stream) {
    return sample_batch(ctx, n, k, x, y, kill_t, t_cut, is_ast, injected, box, log_zoom, budget, sel, qx_out, qy_out,
                        n_sel, stream);
}

namespace {

// Self-test of the sample kernel's grid barrier: block 1 leaves without
// arriving, so block 0's wait runs out after max_polls polls and records
// SSS_ERR_TIMEOUT.
__global__ void k_sample_barrier_selftest(Ctl* ctl, unsigned max_polls, int* status) {
    __shared__ int bad;
    unsigned epoch = 0;
    if (blockIdx.x != 0) return;
    if (!grid_barrier(ctl, epoch, &bad, max_polls) && threadIdx.x == 0)
        atomicCAS(status, SSS_OK, *(volatile int*)&ctl->err);
}

}  // namespace

int sss_stream_barrier_selftest(sss_ctx* ctx, double limit_s, cudaStream_t st) {
    void* scr = nullptr;
    int rc = sss_scratch(ctx, sizeof(Ctl) + 256, &scr);
    if (rc) return rc;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(scr, 0, sizeof(Ctl), st));
    const double polls = limit_s / 32e-9;              // at least 32 ns a poll
    const unsigned max_polls = polls < 1.0 ? 1u : (polls > 4e9 ? 4000000000u : (unsigned)polls);
    k_sample_barrier_selftest<<<2, SAMPLE_THREADS, 0, st>>>((Ctl*)scr, max_polls, ctx->d_status);
    SSS_LAUNCH_CHECK(ctx, "k_sample_barrier_selftest");
    return SSS_OK;
}
