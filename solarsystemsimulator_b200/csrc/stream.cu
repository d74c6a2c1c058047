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
// The bisection resolves 5 halvings per round: the sum is monotone in s
// (every term is, and rounded addition is monotone), so the 31 midpoints of
// the next 5 levels of the halving tree can be summed at once and the 5
// decisions read off them afterwards, each midpoint formed by the same
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

__global__ void k_disp(const float* __restrict__ x, const float* __restrict__ y, long long n, float* __restrict__ qx,
                       float* __restrict__ qy) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float r = hypotf(x[i], y[i]);
    const float sk = r > 1e-9f ? __fdiv_rn(log1pf(r), __fmul_rn(LOG33F, fmaxf(r, 1e-30f))) : 0.0f;
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
//   cull      display coordinates, tier per body (keep = 0), tier counts
//   (plan)    every block reads the tier counts and takes the reference's
//             branch of _lod_auswahl; the plan is uniform over the grid
//   filter    per thinned tier: cell counts (hist), 8 bisection rounds of
//             5 halvings each (group sums, then every block adds the top
//             levels and walks the same decisions), rates, keep decisions
//   emit      per-block kept counts, then each block places its contiguous
//             range of bodies in ascending order
// A barrier wait polls at most BARRIER_POLLS times; when it runs out the
// block records SSS_ERR_TIMEOUT and every block returns at its next barrier.
constexpr int SAMPLE_THREADS = 512;
constexpr int SAMPLE_WARPS = SAMPLE_THREADS / 32;
constexpr unsigned BARRIER_POLLS = 1u << 21;        // about a second with the 32 ns back-off
constexpr int HIST_CHUNK = SAMPLE_THREADS * 4;      // bodies per shared-memory table fill
constexpr int HIST_SLOTS = 2 * HIST_CHUNK;          // 4096: the hash yields 12 bits
constexpr int EMIT_SUB = SAMPLE_THREADS * 4;        // bodies per block scan in the emit phase
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
    int value_over;                                 // more distinct cell counts than the value table holds
    int fast_steps;                                 // halvings decided from the value histogram
    double lohi[2];                                 // the bisection interval after them
};

constexpr int VALUE_SLOTS = 8192;                   // distinct nonzero cell counts (open addressing)
constexpr int VALUE_MAX = 4096;                     // at most this many are sorted by one block

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
    int* counts;                                    // K2 cell counts (cleared in the cull phase)
    double* rate;                                   // K2 rate quads (4 doubles per cell)
    double* part;                                   // 2 x CAND x GROUPS group sums
    long long* blockcnt;                            // gridDim.x
    unsigned* sel;
    unsigned short* ox;
    unsigned short* oy;
    Ctl* ctl;
    int* vkey;                                      // VALUE_SLOTS: count value, -1 empty
    unsigned* vmul;                                 // VALUE_SLOTS: cells holding it
    double* vpre;                                   // 2 VALUE_MAX: prefix sums of the sorted values
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// false: a wait ran out here or in another block (the caller returns)
__device__ __forceinline__ bool grid_barrier(Ctl* ctl, unsigned& epoch, int* s_bad) {
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
            if (polls >= BARRIER_POLLS || *(volatile int*)&ctl->err) {
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
        struct {                                    // bisection: one group's cells
            double c[GROUP_CELLS];
            double w[GROUP_CELLS];
        } g;
    } u;
    double leaf[GROUP_LEAVES][32];
    double tot[32];
    double dred[SAMPLE_WARPS];
    long long red[SAMPLE_WARPS];
    int wcnt[SAMPLE_WARPS];
    int bad;
};

// Cell counts of the bodies whose tier is in mask: each block fills a
// shared-memory open-addressing table from HIST_CHUNK bodies (dense clouds
// put many bodies of a chunk into a few cells) and adds every distinct cell
// to the global counts once. The table has twice the chunk's slots, so a
// probe ends within HIST_SLOTS steps.
__device__ void phase_hist(const SampleArgs& a, const float* qx, const float* qy, int mask, Smem& sm) {
    for (long long c0 = (long long)blockIdx.x * HIST_CHUNK; c0 < a.n; c0 += (long long)gridDim.x * HIST_CHUNK) {
        for (int j = threadIdx.x; j < HIST_SLOTS; j += SAMPLE_THREADS) {
            sm.u.h.key[j] = -1;
            sm.u.h.val[j] = 0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < HIST_CHUNK / SAMPLE_THREADS; ++r) {
            const long long i = c0 + (long long)r * SAMPLE_THREADS + threadIdx.x;
            if (i >= a.n) break;
            const unsigned char t = __ldcg(a.tier + i);
            if (!((mask >> t) & 1)) continue;
            const int c = cell_of(__ldcg(qy + i), a.b.y0, a.b.sy) * K + cell_of(__ldcg(qx + i), a.b.x0, a.b.sx);
            unsigned h = ((unsigned)c * 2654435761u) >> 20;       // Fibonacci hash to 12 bits
            for (int probe = 0; probe < HIST_SLOTS; ++probe) {
                const int prev = atomicCAS(sm.u.h.key + h, -1, c);
                if (prev == -1 || prev == c) {
                    atomicAdd(sm.u.h.val + h, 1);
                    break;
                }
                h = (h + 1) & (HIST_SLOTS - 1);
            }
        }
        __syncthreads();
        for (int j = threadIdx.x; j < HIST_SLOTS; j += SAMPLE_THREADS)
            if (sm.u.h.key[j] >= 0) atomicAdd(a.counts + sm.u.h.key[j], sm.u.h.val[j]);
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
__device__ void phase_group_sums(const SampleArgs& a, double lo, double hi, double* part, Smem& sm) {
    const int leaf = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int g = blockIdx.x; g < GROUPS; g += gridDim.x) {
        constexpr int PER_T = GROUP_CELLS / SAMPLE_THREADS;
        int cv[PER_T];
#pragma unroll
        for (int k = 0; k < PER_T; ++k) cv[k] = __ldcg(a.counts + g * GROUP_CELLS + k * SAMPLE_THREADS + threadIdx.x);
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

__device__ __forceinline__ double block_excl_scan_d(double v, Smem& sm, double* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    __syncthreads();
    if (lane == 31) sm.dred[warp] = inc;
    __syncthreads();
    double before = 0.0, all = 0.0;
#pragma unroll
    for (int w = 0; w < SAMPLE_WARPS; ++w) {
        const double x = sm.dred[w];
        if (w < warp) before += x;
        all += x;
    }
    *total = all;
    return before + (inc - v);
}

__device__ __forceinline__ void value_insert(const SampleArgs& a, int v, unsigned m) {
    unsigned h = ((unsigned)v * 2654435761u) >> 19;                  // Fibonacci hash to 13 bits
    for (int probe = 0; probe < VALUE_SLOTS; ++probe) {
        const int prev = atomicCAS(a.vkey + h, -1, v);
        if (prev == -1 || prev == v) {
            atomicAdd(a.vmul + h, m);
            return;
        }
        h = (h + 1) & (VALUE_SLOTS - 1);
    }
    atomicExch(&a.ctl->value_over, 1);
}
static_assert(VALUE_SLOTS == 1 << 13, "13-bit hash");

// The histogram of the nonzero cell counts (how many cells hold each count):
// each block takes a contiguous range of cells, merges its values in a
// shared-memory table and adds them to the global table. A global table that
// runs out of slots sets value_over (the bisection then takes the exact path).
__device__ void phase_values(const SampleArgs& a, Smem& sm) {
    for (int j = threadIdx.x; j < HIST_SLOTS; j += SAMPLE_THREADS) {
        sm.u.h.key[j] = -1;
        sm.u.h.val[j] = 0;
    }
    __syncthreads();
    const long long per = (K2 + gridDim.x - 1) / gridDim.x;
    const long long c0 = (long long)blockIdx.x * per, c1 = min(c0 + per, (long long)K2);
    for (long long c = c0 + threadIdx.x; c < c1; c += SAMPLE_THREADS) {
        const int v = __ldcg(a.counts + c);
        if (v <= 0) continue;
        unsigned h = ((unsigned)v * 2654435761u) >> 20;              // 12 bits
        bool done = false;
        for (int probe = 0; probe < HIST_SLOTS; ++probe) {
            const int prev = atomicCAS(sm.u.h.key + h, -1, v);
            if (prev == -1 || prev == v) {
                atomicAdd(sm.u.h.val + h, 1);
                done = true;
                break;
            }
            h = (h + 1) & (HIST_SLOTS - 1);
        }
        if (!done) value_insert(a, v, 1u);                           // a full block table: straight to the global one
    }
    __syncthreads();
    for (int j = threadIdx.x; j < HIST_SLOTS; j += SAMPLE_THREADS)
        if (sm.u.h.key[j] >= 0) value_insert(a, sm.u.h.key[j], (unsigned)sm.u.h.val[j]);
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
__device__ void block_fast_bisection(const SampleArgs& a, double budget, Smem& sm) {
    int* sv = sm.u.h.key;                                            // sorted values (VALUE_MAX)
    int* sn = sm.u.h.val;                                            // their cell counts
    static_assert(HIST_SLOTS >= VALUE_MAX, "sort space");
    constexpr int PER = VALUE_SLOTS / SAMPLE_THREADS;
    int cnt = 0;
    for (int q = 0; q < PER; ++q) cnt += __ldcg(a.vkey + threadIdx.x * PER + q) >= 0;
    long long total = 0;
    const long long off = block_excl_scan_ll(cnt, sm, &total);
    if (__ldcg(&a.ctl->value_over) != 0 || total > VALUE_MAX || total < 1) {
        if (threadIdx.x == 0) {
            a.ctl->lohi[0] = 0.0;
            a.ctl->lohi[1] = budget;
            a.ctl->fast_steps = 0;
        }
        return;
    }
    const int D = (int)total;
    int Dp = 1;
    while (Dp < D) Dp <<= 1;
    int w = (int)off;
    for (int q = 0; q < PER; ++q) {
        const int slot = threadIdx.x * PER + q;
        const int v = __ldcg(a.vkey + slot);
        if (v >= 0) {
            sv[w] = v;
            sn[w] = (int)__ldcg(a.vmul + slot);
            ++w;
        }
    }
    for (int i = D + threadIdx.x; i < Dp; i += SAMPLE_THREADS) {
        sv[i] = INT_MAX;
        sn[i] = 0;
    }
    __syncthreads();
    // bitonic sort of (value, cells) by value, ascending (the values are distinct)
    for (int size = 2; size <= Dp; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < Dp / 2; i += SAMPLE_THREADS) {
                const int l = 2 * i - (i & (stride - 1)), r = l + stride;
                const bool up = (l & size) == 0;
                if ((sv[l] > sv[r]) == up) {
                    const int tv = sv[l], tn = sn[l];
                    sv[l] = sv[r];
                    sn[l] = sn[r];
                    sv[r] = tv;
                    sn[r] = tn;
                }
            }
            __syncthreads();
        }
    // prefix sums over chunks of consecutive values, then across the chunks
    const int ch = (D + SAMPLE_THREADS - 1) / SAMPLE_THREADS;
    const int i0 = threadIdx.x * ch, i1 = min(i0 + ch, D);
    double la = 0.0, lw = 0.0;
    for (int i = i0; i < i1; ++i) {
        la += (double)sn[i] * (double)sv[i];
        lw += (double)sn[i] * cell_weight(sv[i]);
    }
    double tot_a = 0.0, tot_w = 0.0;
    double ea = block_excl_scan_d(la, sm, &tot_a);
    double ew = block_excl_scan_d(lw, sm, &tot_w);
    for (int i = i0; i < i1; ++i) {
        a.vpre[2 * i] = ea;
        a.vpre[2 * i + 1] = ew;
        ea += (double)sn[i] * (double)sv[i];
        ew += (double)sn[i] * cell_weight(sv[i]);
    }
    if (threadIdx.x == 0) {
        a.vpre[2 * D] = tot_a;
        a.vpre[2 * D + 1] = tot_w;
    }
    __syncthreads();
    // warp 0: BISECT_D halvings per round, lane c evaluating the midpoint of
    // node c + 1 of the halving tree below (lo, hi) (node_mid: the same
    // arithmetic as the sequential halving), the decisions read off the
    // path by shuffles; the walk stops at the first uncertain node
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const double W = tot_w;
        double lo = 0.0, hi = budget;
        int steps = 0;
        bool stop = false;
        while (steps < 40 && !stop) {
            double F = 0.0, margin = 0.0;
            if (lane < CAND) {
                const double s = node_mid(lane + 1, lo, hi);
                const double s2 = s * s;
                int l = 0, r = D;                                    // k = #values <= s^2
                while (l < r) {
                    const int m = (l + r) >> 1;
                    if ((double)sv[m] <= s2) l = m + 1;
                    else r = m;
                }
                F = a.vpre[2 * l] + s * (W - a.vpre[2 * l + 1]);
                margin = 1e-13 * (F + s * W + budget);
            }
            const int levels = min(BISECT_D, 40 - steps);
            int node = 1;
            for (int d = 0; d < levels; ++d) {
                const double Fn = __shfl_sync(0xffffffffu, F, node - 1);
                const double Mn = __shfl_sync(0xffffffffu, margin, node - 1);
                const double s = __dmul_rn(0.5, __dadd_rn(lo, hi));
                if (Fn > budget + Mn) {
                    hi = s;
                    node = 2 * node;
                } else if (Fn < budget - Mn) {
                    lo = s;
                    node = 2 * node + 1;
                } else {
                    stop = true;
                    break;
                }
                ++steps;
            }
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
// ctl->kept[slot]. Returns false when a barrier gave up.
__device__ bool filter(const SampleArgs& a, const float* qx, const float* qy, int mask, long long budget, int slot,
                       unsigned& epoch, Smem& sm) {
    phase_hist(a, qx, qy, mask, sm);
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    phase_values(a, sm);
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    if (blockIdx.x == 0) block_fast_bisection(a, (double)budget, sm);
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    double lo = __ldcg(&a.ctl->lohi[0]), hi = __ldcg(&a.ctl->lohi[1]);
    // the halvings the histogram could not decide (normally none): exact rounds
    int left = 40 - __ldcg(&a.ctl->fast_steps);
    for (int round = 0; left > 0; ++round) {
        double* part = a.part + (round & 1) * CAND * GROUPS;
        phase_group_sums(a, lo, hi, part, sm);
        if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
        const int levels = min(BISECT_D, left);
        phase_walk(part, (double)budget, lo, hi, levels, sm);
        left -= levels;
    }
    const long long T = (long long)gridDim.x * SAMPLE_THREADS;
    const long long gt = (long long)blockIdx.x * SAMPLE_THREADS + threadIdx.x;
    // rate quad of cell (iy, ix): the rates of (iy, ix), (iy, ix1), (iy1, ix),
    // (iy1, ix1), the four a body's bilinear rate reads, in one 32-byte sector
    for (long long c = gt; c < K2; c += T) {
        const int ix = (int)(c % K), iy = (int)(c / K);
        const int ix1 = min(ix + 1, K - 1), iy1 = min(iy + 1, K - 1);
        const int cells[4] = {iy * K + ix, iy * K + ix1, iy1 * K + ix, iy1 * K + ix1};
        double r[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = __ldcg(a.counts + cells[q]);
            r[q] = k > 0 ? __ddiv_rn(fmin((double)k, __dmul_rn(lo, cell_weight(k))), (double)k) : 0.0;
        }
        double2* dst = (double2*)(a.rate + 4 * c);
        dst[0] = make_double2(r[0], r[1]);
        dst[1] = make_double2(r[2], r[3]);
    }
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return false;
    const unsigned char* __restrict__ tier = a.tier;
    unsigned char* __restrict__ keep = a.keep;
    long long kept = 0;
    for (long long i0 = gt; i0 < a.n; i0 += 2 * T) {
        unsigned char t[2];
        float px[2], py[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const long long i = i0 + u * T;
            t[u] = i < a.n ? __ldcg(tier + i) : 0;
            px[u] = i < a.n ? __ldcg(qx + i) : 0.0f;
            py[u] = i < a.n ? __ldcg(qy + i) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (!((mask >> t[u]) & 1)) continue;
            const long long i = i0 + u * T;
            const float fx = frac_coord(px[u], a.b.x0, a.b.sx), fy = frac_coord(py[u], a.b.y0, a.b.sy);
            const int ix = (int)floorf(fx), iy = (int)floorf(fy);
            const double2* rq = (const double2*)(a.rate + 4 * (iy * K + ix));
            const double2 r0 = __ldcg(rq), r1 = __ldcg(rq + 1);
            const double tx = __dsub_rn((double)fx, (double)ix), ty = __dsub_rn((double)fy, (double)iy);
            const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
            double rp = __dmul_rn(__dmul_rn(r0.x, ux), uy);
            rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(r0.y, tx), uy));
            rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(r1.x, ux), ty));
            rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(r1.y, tx), ty));
            if (index_hash((unsigned long long)i) < rp) {
                keep[i] = 1;
                ++kept;
            }
        }
    }
    // the cell counts are dead now (the rates hold what the keep decisions
    // need): clear them for a following filter
    for (long long c = gt; c < K2; c += T) a.counts[c] = 0;
    for (long long c = gt; c < VALUE_SLOTS; c += T) {
        a.vkey[c] = -1;
        a.vmul[c] = 0;
    }
    if (gt == 0) a.ctl->value_over = 0;
    kept = block_sum_ll(kept, sm.red);
    if (threadIdx.x == 0 && kept) atomicAdd(a.ctl->kept + slot, (unsigned long long)kept);
    return grid_barrier(a.ctl, epoch, &sm.bad);
}

__global__ void __launch_bounds__(SAMPLE_THREADS) k_sample(SampleArgs a) {
    __shared__ Smem sm;
    unsigned epoch = 0;
    const long long T = (long long)gridDim.x * SAMPLE_THREADS;
    const long long gt = (long long)blockIdx.x * SAMPLE_THREADS + threadIdx.x;
    const float* qx = a.log_zoom ? a.qx : a.x;
    const float* qy = a.log_zoom ? a.qy : a.y;
    // ---- cull
    long long n1 = 0, n2 = 0, n3 = 0;
    for (long long c = gt; c < K2; c += T) a.counts[c] = 0;
    for (long long c = gt; c < VALUE_SLOTS; c += T) {
        a.vkey[c] = -1;
        a.vmul[c] = 0;
    }
    if (gt == 0) a.ctl->value_over = 0;
    for (long long i = gt; i < a.n; i += T) {
        float px = a.x[i], py = a.y[i];
        const double kt = a.kill_t[i];
        const unsigned char ast = a.is_ast[i], inj = a.injected ? a.injected[i] : 0;
        if (a.log_zoom) {
            const float r = hypotf(px, py);
            const float sk = r > 1e-9f ? __fdiv_rn(log1pf(r), __fmul_rn(LOG33F, fmaxf(r, 1e-30f))) : 0.0f;
            px = __fmul_rn(px, sk);
            py = __fmul_rn(py, sk);
            a.qx[i] = px;
            a.qy[i] = py;
        }
        unsigned char t = 0;
        if ((kt > a.t_cut) & (px >= a.b.x0) & (px <= a.b.x1) & (py >= a.b.y0) & (py <= a.b.y1))
            t = !ast ? 1 : (inj ? 3 : 2);
        a.tier[i] = t;
        a.keep[i] = 0;
        n1 += t == 1;
        n2 += t == 2;
        n3 += t == 3;
    }
    n1 = block_sum_ll(n1, sm.red);
    n2 = block_sum_ll(n2, sm.red);
    n3 = block_sum_ll(n3, sm.red);
    if (threadIdx.x == 0) {
        if (n1) atomicAdd(a.ctl->tier_cnt + 1, (unsigned long long)n1);
        if (n2) atomicAdd(a.ctl->tier_cnt + 2, (unsigned long long)n2);
        if (n3) atomicAdd(a.ctl->tier_cnt + 3, (unsigned long long)n3);
    }
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return;
    // ---- plan (the reference's _lod_auswahl), identical in every block
    const long long mm = (long long)__ldcg(a.ctl->tier_cnt + 1), ma = (long long)__ldcg(a.ctl->tier_cnt + 2),
                    mi = (long long)__ldcg(a.ctl->tier_cnt + 3);
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
                    kept = (long long)__ldcg(a.ctl->kept + 0);
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
                    kept = (long long)__ldcg(a.ctl->kept + q);
                }
                rest -= kept;
            }
        }
    }
    // ---- emit: block b owns bodies [b * chunk, (b + 1) * chunk)
    const long long chunk = ((a.n + gridDim.x - 1) / gridDim.x + EMIT_SUB - 1) / EMIT_SUB * EMIT_SUB;
    const long long c0 = (long long)blockIdx.x * chunk, c1 = min(c0 + chunk, a.n);
    long long mine = 0;
    for (long long i = c0 + threadIdx.x; i < c1; i += SAMPLE_THREADS)
        mine += __ldcg(a.keep + i) | ((all_mask >> __ldcg(a.tier + i)) & 1);
    mine = block_sum_ll(mine, sm.red);
    if (threadIdx.x == 0) a.blockcnt[blockIdx.x] = mine;
    if (!grid_barrier(a.ctl, epoch, &sm.bad)) return;
    long long before = 0;
    for (int j = threadIdx.x; j < (int)blockIdx.x; j += SAMPLE_THREADS) before += __ldcg(a.blockcnt + j);
    long long off = block_sum_ll(before, sm.red);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long s0 = c0; s0 < c1; s0 += EMIT_SUB) {
        const long long i0 = s0 + (long long)threadIdx.x * 4;
        unsigned bits = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const long long i = i0 + j;
            if (i < c1 && (__ldcg(a.keep + i) | ((all_mask >> __ldcg(a.tier + i)) & 1))) bits |= 1u << j;
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
        for (int j = 0; j < 4; ++j) {
            if (!((bits >> j) & 1)) continue;
            const long long i = i0 + j;
            a.sel[q] = (unsigned)i;
            a.ox[q] = quant(__ldcg(qx + i), a.b.x0, a.b.sx);
            a.oy[q] = quant(__ldcg(qy + i), a.b.y0, a.b.sy);
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
    int* vkey;
    unsigned* vmul;
    double* vpre;
    long long* blockcnt;
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
    const size_t o_cnts = off; off += al((size_t)K2 * 4);
    const size_t o_rate = off; off += al((size_t)K2 * 32);
    const size_t o_part = off; off += al((size_t)2 * CAND * GROUPS * 8);
    const size_t o_vkey = off; off += al((size_t)VALUE_SLOTS * 4);
    const size_t o_vmul = off; off += al((size_t)VALUE_SLOTS * 4);
    const size_t o_vpre = off; off += al((size_t)2 * (VALUE_MAX + 1) * 8);
    const size_t o_blk = off; off += al((size_t)grid * 8);
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
    W->vkey = (int*)(p + o_vkey);
    W->vmul = (unsigned*)(p + o_vmul);
    W->vpre = (double*)(p + o_vpre);
    W->blockcnt = (long long*)(p + o_blk);
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
    a.blockcnt = W.blockcnt;
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
