// Mixed-precision all-pairs self-gravity with the pair distances formed on
// the 5th-generation tensor cores (SSS_PREC_MIXED_TC).
//
// Replaces the pair loop of `beschleunigung` (reference
// backend/selfgrav_kernel.py:222-260) with the same physics: a_i = sum_j
// Gm_j (x_j - x_i) / (|x_j - x_i|^2 + eps^2)^(3/2).
//
// Per tile of TC_TS sources with bounding-box centre C, the target offsets
// o_i = x_i - C and source offsets b_j = x_j - C are formed in f64 and
// rounded once to f32 (the f64 position differences cast to f32 of the
// mixed path). The squared distances of all 128 x 128 pairs of a target
// block and a tile come from one tensor-core product (tcgen05.mma
// kind::tf32, f32 accumulation in tensor memory):
//
//   r^2_ij = -2 o_i . b_j + (|o_i|^2 + eps^2) + |b_j|^2      A1 (128 x 16) x B1^T (16 x 128)
//
// with every f32 operand x split into TF32 parts hi = x with its low 13
// mantissa bits cleared and lo = x - hi, and each cross product formed as
// hi*hi + lo*hi + hi*lo (split TF32, close to an f32 product). The CUDA
// cores read r^2 back (tcgen05.ld) and do the rest of a pair in packed f32x2
// arithmetic, two sources per instruction: s = rsqrt(r^2)^3 (the f32 rsqrt)
// and the four sums S_w = sum_j s_ij w_j of w_j = Gm_j (b_j, 1), 6 FMA-pipe
// operations and one special-function operation per pair against 11 and
// one in the SIMT mixed kernel. A tile's f32 sums are folded into f64
// accumulators per target: a_i += S_xyz,i - o_i S_m,i (the compensated
// split of the mixed path).
//
// The r^2 product loses accuracy when a pair's distance is small against
// the offsets from the tile centre, so a (target block, tile) pair whose
// bounding boxes are closer than TC_KAPPA times the sum of their half
// diagonals takes an f32 pair loop on the CUDA cores instead (about 1 % of
// the tiles on the 262,144-body lattice). Targets and sources are taken in
// Morton order (a device radix sort per evaluation), so the 128 targets of a
// CTA and the 128 sources of a tile are compact.
//
// CTA = 128 threads = the 128 TMEM lanes, two targets per thread (target
// groups 0 and 1, one r^2 product each): thread t owns row t of both. The
// r^2 of a 32-source unit for both groups is double buffered in tensor
// memory (128 columns per CTA, four CTAs per SM); the operands of tile f + 1
// (the A1 rows of the thread's targets, the B1 row and weights of the
// thread's source) are built in shared memory while tile f runs. One thread
// issues the MMAs and commits them to mbarriers; every wait is bounded
// (SSS_ERR_TIMEOUT).
//
// Measured on the 262,144-source benchmark state: 79.0 ms per force
// evaluation with the sorts and the tile prep (the SIMT mixed kernel:
// 75.8 ms), median relative force error 1.4e-7 against f64.

#include "allpairs.cuh"
#include "devscan.cuh"

namespace {

using sss_ap::Epi;

constexpr int TC_NT = 128;                 // threads per CTA = TMEM lanes
constexpr int TC_TPT = 2;                  // targets per thread (one per target group)
constexpr int TC_TB = TC_NT * TC_TPT;      // targets per CTA
constexpr int TC_TS = 128;                 // sources per tile (one centre)
constexpr int TC_US = 32;                  // sources per unit = N of one r^2 product
constexpr int TC_UPT = TC_TS / TC_US;      // units per tile
static_assert(TC_US == 32, "a unit is summed as two halves of 16 sources");
constexpr int TC_K1 = 16;                  // K of the r^2 product (13 used)
constexpr int TC_MAXLIST = 1024;           // tiles per chunk
constexpr double TC_KAPPA = 0.25;          // near test: box gap <= kappa * (half diagonals)
constexpr int TC_WAVES = 16;
constexpr int TC_MINB = 4;                 // CTAs per SM

// tensor memory: r^2 of a unit for both target groups, double buffered
constexpr uint32_t COL_D1 = 0;                           // [2 buffers][2 groups][TC_US]
constexpr uint32_t TMEM_COLS = 2 * TC_TPT * TC_US;
static_assert(TMEM_COLS * TC_MINB <= 512, "the CTAs of an SM share its 512 TMEM columns");

// shared memory (bytes); MMA operands in the canonical no-swizzle K-major layout
constexpr int A1_BYTES = TC_NT * TC_K1 * 4;             // one target group x K1
constexpr int B1_BYTES = TC_TS * TC_K1 * 4;             // sources x K1
constexpr int W_BYTES = TC_TS * 16;                     // source weights, pair-interleaved
constexpr int OFF_A1 = 0;                               // [2 tile parity][2 groups]
constexpr int OFF_B1 = OFF_A1 + 2 * TC_TPT * A1_BYTES;  // [2 tile parity]
constexpr int OFF_W = OFF_B1 + 2 * B1_BYTES;            // [2 tile parity]
constexpr int OFF_LIST = OFF_W + 2 * W_BYTES;           // uint16 [TC_MAXLIST] far | near tiles
constexpr int OFF_BAR = OFF_LIST + TC_MAXLIST * 2;      // mbarriers m1[2], end; TMEM slot
constexpr int OFF_NEAR = OFF_A1;                        // float4 [TC_TS] near-tile sources (after the far loop)
constexpr int SMEM_BYTES = OFF_BAR + 64;
static_assert(TC_MINB * (SMEM_BYTES + 2048) <= 228 * 1024, "shared memory for TC_MINB CTAs per SM");
static_assert((TC_MINB + 1) * (SMEM_BYTES + 1024) > 228 * 1024, "no more CTAs per SM than TMEM holds");

// ------------------------------------------------------------ tcgen05 pieces

// byte offset of element (r, k) of a canonical K-major operand of 32-bit
// elements with K columns: core matrices of 8 rows x 16 bytes, K-adjacent
// core matrices 128 bytes apart, 8-row groups K * 32 bytes apart
__device__ __forceinline__ int canon32(int r, int k, int K) {
    return ((r >> 3) * (K >> 2) + (k >> 2)) * 128 + (r & 7) * 16 + (k & 3) * 4;
}
// shared-memory matrix descriptor of that layout (version 1, no swizzle)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int K) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)((K * 32) >> 4) << 32) | (1ull << 46);
}
// kind::tf32 instruction descriptor: D f32, A and B TF32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] B[smem]^T
__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t da, uint64_t db, uint32_t id, int acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d), "l"(da), "l"(db), "r"(id), "r"(acc) : "memory");
}
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(sss_smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void ld16(uint32_t addr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(sss_smem_addr(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(cols) : "memory");
}

// TF32 split: hi keeps the top 11 significant bits, lo = x - hi (exact)
__device__ __forceinline__ float tf_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xffffe000u); }
__device__ __forceinline__ float4 f4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }

// packed f32x2 arithmetic (two sources per instruction)
typedef unsigned long long f2x;
__device__ __forceinline__ f2x pk2(float lo, float hi) {
    return (f2x)__float_as_uint(lo) | ((f2x)__float_as_uint(hi) << 32);
}
__device__ __forceinline__ void upk2(f2x v, float& lo, float& hi) {
    lo = __uint_as_float((unsigned)v);
    hi = __uint_as_float((unsigned)(v >> 32));
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
    f2x d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
    f2x d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// ------------------------------------------------------------ Morton order

// order-preserving map of f64 onto u64 (for atomicMin / atomicMax)
__device__ __forceinline__ unsigned long long ord64(double x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | (1ull << 63));
}
__device__ __forceinline__ double unord64(unsigned long long u) {
    return __longlong_as_double((long long)((u >> 63) ? (u & ~(1ull << 63)) : ~u));
}

// box[0..2] = min x, y, z; box[3..5] = max (order-mapped; preset to the
// identities by the caller)
template <int D>
__global__ void __launch_bounds__(256) k_tc_bbox(const double4* __restrict__ pos, int64_t n,
                                                 unsigned long long* __restrict__ box) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 p = pos[i];
        lo[0] = fmin(lo[0], p.x); hi[0] = fmax(hi[0], p.x);
        lo[1] = fmin(lo[1], p.y); hi[1] = fmax(hi[1], p.y);
        const double z = (D == 3) ? p.z : 0.0;
        lo[2] = fmin(lo[2], z); hi[2] = fmax(hi[2], z);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    if ((threadIdx.x & 31) == 0 && lo[0] <= hi[0]) {
        for (int c = 0; c < 3; ++c) {
            atomicMin(&box[c], ord64(lo[c]));
            atomicMax(&box[3 + c], ord64(hi[c]));
        }
    }
}

__device__ __forceinline__ unsigned long long spread3(unsigned v) {   // 10 bits -> every third bit
    unsigned long long x = v & 0x3ffu;
    x = (x | (x << 16)) & 0x030000FFull;
    x = (x | (x << 8)) & 0x0300F00Full;
    x = (x | (x << 4)) & 0x030C30C3ull;
    x = (x | (x << 2)) & 0x09249249ull;
    return x;
}

// 30-bit Morton key of each body on a 1024^3 grid over the box; val = index
template <int D>
__global__ void __launch_bounds__(256) k_tc_morton(const double4* __restrict__ pos, int64_t n,
                                                   const unsigned long long* __restrict__ box,
                                                   unsigned long long* __restrict__ key, unsigned* __restrict__ val) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = pos[i];
    const double c[3] = {p.x, p.y, (D == 3) ? p.z : 0.0};
    unsigned q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double lo = unord64(box[k]), hi = unord64(box[3 + k]);
        const double ext = hi - lo;
        const double u = ext > 0.0 ? (c[k] - lo) * (1023.999 / ext) : 0.0;
        q[k] = (unsigned)fmin(fmax(u, 0.0), 1023.0);
    }
    key[i] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
    val[i] = (unsigned)i;
}

// One CTA per tile of TC_TS sources in Morton order: bounding box, centre,
// and every source's f32 offset from the centre with its Gm (padding
// entries are zeros: at the centre, massless).
template <int D>
__global__ void __launch_bounds__(TC_TS) k_tc_prep(const double4* __restrict__ src, int64_t n_src,
                                                   const unsigned* __restrict__ sperm, float4* __restrict__ tdat,
                                                   double4* __restrict__ tcen, float4* __restrict__ thalf) {
    __shared__ double red[6][TC_TS / 32];
    const int t = blockIdx.x, j = threadIdx.x;
    const int64_t g = (int64_t)t * TC_TS + j;
    const bool valid = g < n_src;
    double4 s = make_double4(0.0, 0.0, 0.0, 0.0);
    if (valid) {
        s = src[sperm[g]];
        if (D == 2) s.z = 0.0;
    }
    double lo[3] = {valid ? s.x : 1e300, valid ? s.y : 1e300, valid ? s.z : 1e300};
    double hi[3] = {valid ? s.x : -1e300, valid ? s.y : -1e300, valid ? s.z : -1e300};
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    if ((j & 31) == 0)
        for (int c = 0; c < 3; ++c) { red[c][j >> 5] = lo[c]; red[3 + c][j >> 5] = hi[c]; }
    __syncthreads();
    double cen[3], half[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double l = red[c][0], h = red[3 + c][0];
        for (int w = 1; w < TC_TS / 32; ++w) { l = fmin(l, red[c][w]); h = fmax(h, red[3 + c][w]); }
        cen[c] = 0.5 * (l + h);
        half[c] = 0.5 * (h - l);
    }
    tdat[g] = valid ? make_float4(__double2float_rn(s.x - cen[0]), __double2float_rn(s.y - cen[1]),
                                  __double2float_rn(s.z - cen[2]), __double2float_rn(s.w))
                    : make_float4(0.f, 0.f, 0.f, 0.f);
    if (j == 0) {
        const double diag = sqrt(half[0] * half[0] + half[1] * half[1] + half[2] * half[2]);
        tcen[t] = make_double4(cen[0], cen[1], cen[2], diag * (1.0 + 1e-12));
        thalf[t] = make_float4(__double2float_ru(half[0]), __double2float_ru(half[1]), __double2float_ru(half[2]), 0.f);
    }
}

// ------------------------------------------------------------ force kernel

struct TcArgs {
    const float4* tdat;       // [n_tiles * TC_TS] {bx, by, bz, Gm}: f32 offsets from the tile centre
    const double4* tcen;      // [n_tiles] {cx, cy, cz, half diagonal}
    const float4* thalf;      // [n_tiles] half extents (rounded up)
    int n_tiles, n_chunks, tiles_per_chunk;
    const double4* tgt;
    int64_t n_tgt;
    const unsigned* tperm;    // [n_slots] target of each slot, >= n_tgt for none
    int64_t n_slots;
    float eps2f;
    double4* part;            // [n_chunks][n_slots] chunk partial sums (n_chunks > 1)
    unsigned* counters;       // [n_tblocks]
    int* status;
    Epi epi;
};

// 16 sources of the current tile against the thread's two targets: r^2
// from tensor memory (ra: target group 0, rb: group 1), weights
// (pair-interleaved {wx wx' wy wy'}, {wz wz' wm wm'}) from shared memory,
// sums into the packed accumulators of each target
__device__ __forceinline__ void pairs16(const float (&ra)[16], const float (&rb)[16],
                                        const ulonglong2* __restrict__ w, f2x (&sa)[4], f2x (&sb)[4]) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const ulonglong2 wxy = w[2 * q], wzm = w[2 * q + 1];
        const f2x ia = pk2(sss_rsqrt_approx_f32(ra[2 * q]), sss_rsqrt_approx_f32(ra[2 * q + 1]));
        const f2x ib = pk2(sss_rsqrt_approx_f32(rb[2 * q]), sss_rsqrt_approx_f32(rb[2 * q + 1]));
        const f2x ga = mul2(ia, mul2(ia, ia));
        const f2x gb = mul2(ib, mul2(ib, ib));
        sa[0] = fma2(ga, wxy.x, sa[0]);
        sb[0] = fma2(gb, wxy.x, sb[0]);
        sa[1] = fma2(ga, wxy.y, sa[1]);
        sb[1] = fma2(gb, wxy.y, sb[1]);
        sa[2] = fma2(ga, wzm.x, sa[2]);
        sb[2] = fma2(gb, wzm.x, sb[2]);
        sa[3] = fma2(ga, wzm.y, sa[3]);
        sb[3] = fma2(gb, wzm.y, sb[3]);
    }
}

__device__ __forceinline__ double lanes_sum(f2x v) {
    float l0, l1;
    upk2(v, l0, l1);
    return (double)l0 + (double)l1;
}

template <int D>
__global__ void __launch_bounds__(TC_NT, TC_MINB) k_force_tc(const TcArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ double s_box[TC_NT / 32][6];
    __shared__ double s_cen[2][3];     // centres of the far tiles in flight, by tile parity
    __shared__ int s_cnt[TC_NT / 32][2];
    __shared__ unsigned s_last;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tb = blockIdx.x / a.n_chunks;
    const int ch = blockIdx.x - tb * a.n_chunks;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + OFF_BAR);     // m1[2], end
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + OFF_BAR + 32);
    uint16_t* list = reinterpret_cast<uint16_t*>(smem + OFF_LIST);

    // the thread's targets: slot tid of target group 0 and of group 1
    int64_t slot[TC_TPT];
    unsigned ti[TC_TPT];
    bool has[TC_TPT];
    double3 p[TC_TPT];
#pragma unroll
    for (int g = 0; g < TC_TPT; ++g) {
        slot[g] = (int64_t)tb * TC_TB + g * TC_NT + tid;
        ti[g] = a.tperm[slot[g]];
        has[g] = (int64_t)ti[g] < a.n_tgt;
        const double4 q = has[g] ? a.tgt[ti[g]] : make_double4(0.0, 0.0, 0.0, 0.0);
        p[g] = make_double3(q.x, q.y, (D == 3) ? q.z : 0.0);
    }

    if (tid == 0) {
        for (int q = 0; q < 3; ++q) sss_mbar_init(&bar[q], 1);
        sss_fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tslot, TMEM_COLS);

    // bounding box of the CTA's targets
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
#pragma unroll
    for (int g = 0; g < TC_TPT; ++g)
        if (has[g]) {
            lo[0] = fmin(lo[0], p[g].x); hi[0] = fmax(hi[0], p[g].x);
            lo[1] = fmin(lo[1], p[g].y); hi[1] = fmax(hi[1], p[g].y);
            lo[2] = fmin(lo[2], p[g].z); hi[2] = fmax(hi[2], p[g].z);
        }
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    if (lane == 0)
        for (int c = 0; c < 3; ++c) { s_box[warp][c] = lo[c]; s_box[warp][3 + c] = hi[c]; }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;
    double bc[3], bh[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double l = s_box[0][c], h = s_box[0][3 + c];
        for (int w = 1; w < TC_NT / 32; ++w) { l = fmin(l, s_box[w][c]); h = fmax(h, s_box[w][3 + c]); }
        bc[c] = 0.5 * (l + h);
        bh[c] = 0.5 * (h - l);
    }
    const double brad = sqrt(bh[0] * bh[0] + bh[1] * bh[1] + bh[2] * bh[2]);

    // classify the chunk's tiles: far ones (tensor cores) to the front of the
    // list in ascending order, near ones (CUDA cores) to the back
    const int t_begin = ch * a.tiles_per_chunk;
    const int t_end = min(t_begin + a.tiles_per_chunk, a.n_tiles);
    const int nt = t_end - t_begin;
    int nfar = 0, nnear = 0;
    for (int base = 0; base < nt; base += TC_NT) {
        const int t = base + tid;
        const bool valid = t < nt;
        bool near = false;
        if (valid) {
            const double4 c = a.tcen[t_begin + t];
            const float4 h = a.thalf[t_begin + t];
            const double gx = fmax(0.0, fabs(c.x - bc[0]) - ((double)h.x + bh[0]));
            const double gy = fmax(0.0, fabs(c.y - bc[1]) - ((double)h.y + bh[1]));
            const double gz = fmax(0.0, fabs(c.z - bc[2]) - ((double)h.z + bh[2]));
            near = sqrt(gx * gx + gy * gy + gz * gz) <= TC_KAPPA * (c.w + brad);
        }
        const unsigned mf = __ballot_sync(0xffffffffu, valid && !near);
        const unsigned mn = __ballot_sync(0xffffffffu, valid && near);
        if (lane == 0) { s_cnt[warp][0] = __popc(mf); s_cnt[warp][1] = __popc(mn); }
        __syncthreads();
        int of = nfar, on = nnear, tf = 0, tn = 0;
        for (int w = 0; w < TC_NT / 32; ++w) {
            if (w < warp) { of += s_cnt[w][0]; on += s_cnt[w][1]; }
            tf += s_cnt[w][0];
            tn += s_cnt[w][1];
        }
        const unsigned below = (1u << lane) - 1u;
        if (valid && !near) list[of + __popc(mf & below)] = (uint16_t)t;
        if (valid && near) list[TC_MAXLIST - 1 - (on + __popc(mn & below))] = (uint16_t)t;
        nfar += tf;
        nnear += tn;
        __syncthreads();
    }

    const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);   // this thread's TMEM lane
    const uint32_t sA1 = sss_smem_addr(smem + OFF_A1), sB1 = sss_smem_addr(smem + OFF_B1);
    constexpr uint32_t ID1 = idesc_tf32(TC_US);
    const float eps2f = a.eps2f;
    double acc[TC_TPT][3];
#pragma unroll
    for (int g = 0; g < TC_TPT; ++g)
        for (int c = 0; c < 3; ++c) acc[g][c] = 0.0;
    bool bad = false, aborted = false;

    // operands of far tile f (parity f & 1): the thread's target rows of A1
    // (one per target group), its source's row of B1 and its weights
    auto fetch = [&](int f, float4& src, double4& c) {
        const int t = t_begin + list[f];
        src = a.tdat[(int64_t)t * TC_TS + tid];
        c = a.tcen[t];
    };
    auto build = [&](int f, const float4& src, const double4& c) {
        const int par = f & 1;
        if (tid == 0) { s_cen[par][0] = c.x; s_cen[par][1] = c.y; s_cen[par][2] = c.z; }
#pragma unroll
        for (int g = 0; g < TC_TPT; ++g) {
            const double o0 = p[g].x - c.x, o1 = p[g].y - c.y, o2 = p[g].z - c.z;
            const float fx = __double2float_rn(o0), fy = __double2float_rn(o1), fz = __double2float_rn(o2);
            const float nn = fmaf(fx, fx, fmaf(fy, fy, fmaf(fz, fz, eps2f)));
            const float gx = -2.f * fx, gy = -2.f * fy, gz = -2.f * fz;
            const float gxh = tf_hi(gx), gyh = tf_hi(gy), gzh = tf_hi(gz), nh = tf_hi(nn);
            uint8_t* ra = smem + OFF_A1 + (par * TC_TPT + g) * A1_BYTES;
            *reinterpret_cast<float4*>(ra + canon32(tid, 0, TC_K1)) = f4(gxh, gx - gxh, gxh, gyh);
            *reinterpret_cast<float4*>(ra + canon32(tid, 4, TC_K1)) = f4(gy - gyh, gyh, gzh, gz - gzh);
            *reinterpret_cast<float4*>(ra + canon32(tid, 8, TC_K1)) = f4(gzh, nh, nn - nh, 1.f);
            *reinterpret_cast<float4*>(ra + canon32(tid, 12, TC_K1)) = f4(1.f, 0.f, 0.f, 0.f);
        }
        const float bx = src.x, by = src.y, bz = src.z, gm = src.w;
        const float q = fmaf(bx, bx, fmaf(by, by, bz * bz));
        const float bxh = tf_hi(bx), byh = tf_hi(by), bzh = tf_hi(bz), qh = tf_hi(q);
        uint8_t* rb = smem + OFF_B1 + par * B1_BYTES;
        *reinterpret_cast<float4*>(rb + canon32(tid, 0, TC_K1)) = f4(bxh, bxh, bx - bxh, byh);
        *reinterpret_cast<float4*>(rb + canon32(tid, 4, TC_K1)) = f4(byh, by - byh, bzh, bzh);
        *reinterpret_cast<float4*>(rb + canon32(tid, 8, TC_K1)) = f4(bz - bzh, 1.f, 1.f, qh);
        *reinterpret_cast<float4*>(rb + canon32(tid, 12, TC_K1)) = f4(q - qh, 0.f, 0.f, 0.f);
        float* rw = reinterpret_cast<float*>(smem + OFF_W + par * W_BYTES) + (tid >> 1) * 8 + (tid & 1);
        rw[0] = gm * bx;
        rw[2] = gm * by;
        rw[4] = gm * bz;
        rw[6] = gm;
    };
    // products of unit u = sources [TC_US (u % TC_UPT), +TC_US) of far tile
    // u / TC_UPT, both target groups, into D1[u & 1]
    auto issue_r2 = [&](int u) {
        const int par = (u / TC_UPT) & 1, q = u % TC_UPT;
        const uint32_t sb = sB1 + par * B1_BYTES + q * (TC_US / 8) * (TC_K1 * 32);
#pragma unroll
        for (int g = 0; g < TC_TPT; ++g) {
            const uint32_t d = tmem + COL_D1 + (u & 1) * (TC_TPT * TC_US) + g * TC_US;
            const uint32_t sa = sA1 + (par * TC_TPT + g) * A1_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_K1 / 8; ++kk)
                mma_ss(d, sdesc(sa + kk * 256, TC_K1), sdesc(sb + kk * 256, TC_K1), ID1, kk);
        }
        commit(&bar[u & 1]);
    };

    const int U = TC_UPT * nfar;
    float4 nsrc = make_float4(0.f, 0.f, 0.f, 0.f);
    double4 ncen = make_double4(0.0, 0.0, 0.0, 0.0);
    if (nfar > 0) {
        fetch(0, nsrc, ncen);
        build(0, nsrc, ncen);
        fence_proxy_async();
        fence_before();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            issue_r2(0);
            issue_r2(1);
        }
    }
    f2x sa[4] = {0ull, 0ull, 0ull, 0ull}, sb[4] = {0ull, 0ull, 0ull, 0ull};
    for (int u = 0; u < U; ++u) {
        const int f = u / TC_UPT, q = u % TC_UPT, b = u & 1, par = f & 1;
        if (q == 0 && f + 1 < nfar) fetch(f + 1, nsrc, ncen);   // in flight while tile f is summed
        bad |= !sss_mbar_wait_bounded(&bar[b], (u >> 1) & 1, a.status);
        fence_after();
        {   // the second half's r^2 loads run while the first half is summed
            float ra0[16], rb0[16], ra1[16], rb1[16];
            const uint32_t col = trow + COL_D1 + b * (TC_TPT * TC_US);
            const ulonglong2* w = reinterpret_cast<const ulonglong2*>(smem + OFF_W + par * W_BYTES) + q * TC_US;
            ld16(col, ra0);
            ld16(col + TC_US, rb0);
            wait_ld();
            ld16(col + 16, ra1);
            ld16(col + TC_US + 16, rb1);
            pairs16(ra0, rb0, w, sa, sb);
            wait_ld();
            pairs16(ra1, rb1, w + 16, sa, sb);
        }
        if (q == TC_UPT - 1) {   // fold the tile's f32 sums into f64: a += S_xyz - o S_m
            const double ma = lanes_sum(sa[3]), mb = lanes_sum(sb[3]);
            const double cx = s_cen[par][0], cy = s_cen[par][1], cz = s_cen[par][2];
            acc[0][0] += lanes_sum(sa[0]) - (p[0].x - cx) * ma;
            acc[0][1] += lanes_sum(sa[1]) - (p[0].y - cy) * ma;
            acc[0][2] += lanes_sum(sa[2]) - (p[0].z - cz) * ma;
            acc[1][0] += lanes_sum(sb[0]) - (p[1].x - cx) * mb;
            acc[1][1] += lanes_sum(sb[1]) - (p[1].y - cy) * mb;
            acc[1][2] += lanes_sum(sb[2]) - (p[1].z - cz) * mb;
#pragma unroll
            for (int k = 0; k < 4; ++k) { sa[k] = 0ull; sb[k] = 0ull; }
        }
        // tile f + 1 into the buffers of tile f - 1 (its products are complete,
        // its weights were read before an earlier barrier); its first unit is
        // issued at this unit's barrier
        const bool next = (q == TC_UPT - 2) && (f + 1 < nfar);
        if (next) {
            build(f + 1, nsrc, ncen);
            fence_proxy_async();
        }
        fence_before();
        if (__syncthreads_or(bad)) { aborted = true; break; }
        if (tid == 0 && u + 2 < U) {
            fence_after();
            issue_r2(u + 2);
        }
    }
    if (nfar > 0) {   // every product issued by thread 0 is complete once this commit arrives
        if (tid == 0) commit(&bar[2]);
        if (!sss_mbar_wait_bounded(&bar[2], 0, a.status)) aborted = true;
        fence_after();
    }

    // near tiles: the f32 pair loop of the mixed kernel
    float4* stage = reinterpret_cast<float4*>(smem + OFF_NEAR);   // the A1 buffers are free now
    for (int k = 0; k < nnear; ++k) {
        const int t = t_begin + list[TC_MAXLIST - 1 - k];
        __syncthreads();
        stage[tid] = a.tdat[(int64_t)t * TC_TS + tid];
        const double4 c = a.tcen[t];
        __syncthreads();
        float ox[TC_TPT], oy[TC_TPT], oz[TC_TPT], sx[TC_TPT], sy[TC_TPT], sz[TC_TPT];
#pragma unroll
        for (int g = 0; g < TC_TPT; ++g) {
            ox[g] = __double2float_rn(p[g].x - c.x);
            oy[g] = __double2float_rn(p[g].y - c.y);
            oz[g] = __double2float_rn(p[g].z - c.z);
            sx[g] = sy[g] = sz[g] = 0.f;
        }
#pragma unroll 4
        for (int j = 0; j < TC_TS; ++j) {
            const float4 s = stage[j];
#pragma unroll
            for (int g = 0; g < TC_TPT; ++g) {
                const float dx = s.x - ox[g], dy = s.y - oy[g], dz = s.z - oz[g];
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2f)));
                const float iv = sss_rsqrt_approx_f32(r2);
                const float q = s.w * (iv * iv * iv);
                sx[g] = fmaf(q, dx, sx[g]);
                sy[g] = fmaf(q, dy, sy[g]);
                sz[g] = fmaf(q, dz, sz[g]);
            }
        }
#pragma unroll
        for (int g = 0; g < TC_TPT; ++g) {
            acc[g][0] += (double)sx[g];
            acc[g][1] += (double)sy[g];
            acc[g][2] += (double)sz[g];
        }
    }

    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
    (void)aborted;

    if (a.n_chunks == 1) {
#pragma unroll
        for (int g = 0; g < TC_TPT; ++g)
            if (has[g]) sss_ap::epilogue<D>(a.epi, ti[g], acc[g][0], acc[g][1], acc[g][2], a.tgt[ti[g]]);
        return;
    }
#pragma unroll
    for (int g = 0; g < TC_TPT; ++g) {
        double2* q = reinterpret_cast<double2*>(a.part + (int64_t)ch * a.n_slots + slot[g]);
        __stcg(q, make_double2(acc[g][0], acc[g][1]));
        __stcg(q + 1, make_double2(acc[g][2], 0.0));
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const unsigned prev = atomicAdd(&a.counters[tb], 1u);
        s_last = (prev == (unsigned)(a.n_chunks - 1)) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int g = 0; g < TC_TPT; ++g) {
        if (!has[g]) continue;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int c = 0; c < a.n_chunks; ++c) {
            const double2* q = reinterpret_cast<const double2*>(a.part + (int64_t)c * a.n_slots + slot[g]);
            const double2 q0 = __ldcg(q), q1 = __ldcg(q + 1);
            sx += q0.x;
            sy += q0.y;
            sz += q1.x;
        }
        sss_ap::epilogue<D>(a.epi, ti[g], sx, sy, sz, a.tgt[ti[g]]);
    }
    if (tid == 0) a.counters[tb] = 0u;   // ready for the next launch
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

namespace sss_ap {

int force_eval_tc(sss_ctx* ctx, int dim, const double4* src, int64_t n_src, const double4* tgt, int64_t n_tgt,
                  double eps2, const Epi& epi, cudaStream_t s) {
    if (!(eps2 > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "SSS_PREC_MIXED_TC needs eps2 > 0");
    if (n_src > ((int64_t)1 << 30) || n_tgt > ((int64_t)1 << 30))
        return sss_set_err(ctx, SSS_ERR_ARG, "SSS_PREC_MIXED_TC: at most 2^30 sources and targets");
    const int n_tiles = (int)((n_src + TC_TS - 1) / TC_TS);
    const int64_t n_tblocks = (n_tgt + TC_TB - 1) / TC_TB;
    const int64_t n_slots = n_tblocks * TC_TB;

    auto kfn = (dim == 3) ? (void*)k_force_tc<3> : (void*)k_force_tc<2>;
    const int key = 6 + (dim == 3);
    if (ctx->occ[key] == 0) {
        SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        int per_sm = 0;
        SSS_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, TC_NT, SMEM_BYTES));
        ctx->occ[key] = per_sm < 1 ? 1 : per_sm;
    }
    // source chunks: enough CTAs for TC_WAVES waves, at most TC_MAXLIST tiles per chunk
    const int64_t want = (int64_t)TC_WAVES * ctx->occ[key] * ctx->num_sms;
    int64_t sc = (want + n_tblocks - 1) / n_tblocks;
    const int64_t sc_min = (n_tiles + TC_MAXLIST - 1) / TC_MAXLIST;
    if (sc < sc_min) sc = sc_min;
    if (sc > n_tiles) sc = n_tiles;
    const int tiles_per_chunk = (int)((n_tiles + sc - 1) / sc);
    const int n_chunks = (n_tiles + tiles_per_chunk - 1) / tiles_per_chunk;
    if (n_tblocks * n_chunks >= ((int64_t)1 << 31))
        return sss_set_err(ctx, SSS_ERR_ARG, "SSS_PREC_MIXED_TC: grid too large");

    // scratch: tiles, centres, half extents, two boxes, sort buffers, partials
    const int64_t nmax = n_src > n_tgt ? n_src : n_tgt;
    size_t off = 0;
    const size_t o_tdat = off; off += al256((size_t)n_tiles * TC_TS * sizeof(float4));
    const size_t o_tcen = off; off += al256((size_t)n_tiles * sizeof(double4));
    const size_t o_thalf = off; off += al256((size_t)n_tiles * sizeof(float4));
    const size_t o_box = off; off += al256(12 * sizeof(unsigned long long));
    const size_t o_sk0 = off; off += al256((size_t)n_src * 8);
    const size_t o_sk1 = off; off += al256((size_t)n_src * 8);
    const size_t o_sv0 = off; off += al256((size_t)n_src * 4);
    const size_t o_sv1 = off; off += al256((size_t)n_src * 4);
    const size_t o_tk0 = off; off += al256((size_t)n_tgt * 8);
    const size_t o_tk1 = off; off += al256((size_t)n_tgt * 8);
    const size_t o_tv0 = off; off += al256((size_t)n_slots * 4);
    const size_t o_tv1 = off; off += al256((size_t)n_tgt * 4);
    const size_t o_rs = off; off += al256(sss_dev::radix_scratch(nmax) * sizeof(long long));
    const size_t o_part = off; off += n_chunks > 1 ? al256((size_t)n_chunks * n_slots * sizeof(double4)) : 0;
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* base = (char*)scr;
    unsigned long long* box = (unsigned long long*)(base + o_box);
    unsigned long long* sk0 = (unsigned long long*)(base + o_sk0);
    unsigned long long* sk1 = (unsigned long long*)(base + o_sk1);
    unsigned* sv0 = (unsigned*)(base + o_sv0);
    unsigned* sv1 = (unsigned*)(base + o_sv1);
    unsigned long long* tk0 = (unsigned long long*)(base + o_tk0);
    unsigned long long* tk1 = (unsigned long long*)(base + o_tk1);
    unsigned* tv0 = (unsigned*)(base + o_tv0);
    unsigned* tv1 = (unsigned*)(base + o_tv1);
    long long* rs = (long long*)(base + o_rs);

    TcArgs a;
    memset(&a, 0, sizeof(a));
    a.tdat = (const float4*)(base + o_tdat);
    a.tcen = (const double4*)(base + o_tcen);
    a.thalf = (const float4*)(base + o_thalf);
    a.n_tiles = n_tiles;
    a.n_chunks = n_chunks;
    a.tiles_per_chunk = tiles_per_chunk;
    a.tgt = tgt;
    a.n_tgt = n_tgt;
    a.tperm = tv0;
    a.n_slots = n_slots;
    a.eps2f = (float)eps2;
    a.status = ctx->d_status;
    a.epi = epi;
    if (n_chunks > 1) {
        a.part = (double4*)(base + o_part);
        rc = sss_counters(ctx, (size_t)n_tblocks, &a.counters);
        if (rc) return rc;
    }

    // Morton order of sources and targets
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(box, 0xff, 3 * sizeof(unsigned long long), s));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(box + 3, 0, 3 * sizeof(unsigned long long), s));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(box + 6, 0xff, 3 * sizeof(unsigned long long), s));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(box + 9, 0, 3 * sizeof(unsigned long long), s));
    if (n_slots > n_tgt)
        SSS_CUDA_TRY(ctx, cudaMemsetAsync(tv0 + n_tgt, 0xff, (size_t)(n_slots - n_tgt) * 4, s));
    const unsigned gb_s = (unsigned)(n_src < 256 * 1184 ? (n_src + 255) / 256 : 1184);
    const unsigned gb_t = (unsigned)(n_tgt < 256 * 1184 ? (n_tgt + 255) / 256 : 1184);
    if (dim == 3) {
        k_tc_bbox<3><<<gb_s, 256, 0, s>>>(src, n_src, box);
        k_tc_bbox<3><<<gb_t, 256, 0, s>>>(tgt, n_tgt, box + 6);
        k_tc_morton<3><<<(unsigned)((n_src + 255) / 256), 256, 0, s>>>(src, n_src, box, sk0, sv0);
        k_tc_morton<3><<<(unsigned)((n_tgt + 255) / 256), 256, 0, s>>>(tgt, n_tgt, box + 6, tk0, tv0);
    } else {
        k_tc_bbox<2><<<gb_s, 256, 0, s>>>(src, n_src, box);
        k_tc_bbox<2><<<gb_t, 256, 0, s>>>(tgt, n_tgt, box + 6);
        k_tc_morton<2><<<(unsigned)((n_src + 255) / 256), 256, 0, s>>>(src, n_src, box, sk0, sv0);
        k_tc_morton<2><<<(unsigned)((n_tgt + 255) / 256), 256, 0, s>>>(tgt, n_tgt, box + 6, tk0, tv0);
    }
    SSS_LAUNCH_CHECK(ctx, "Morton keys");
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(sk0, sv0, sk1, sv1, n_src, rs, s, ctx->d_status, 30));
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(tk0, tv0, tk1, tv1, n_tgt, rs, s, ctx->d_status, 30));
    if (dim == 3)
        k_tc_prep<3><<<n_tiles, TC_TS, 0, s>>>(src, n_src, sv0, (float4*)a.tdat, (double4*)a.tcen, (float4*)a.thalf);
    else
        k_tc_prep<2><<<n_tiles, TC_TS, 0, s>>>(src, n_src, sv0, (float4*)a.tdat, (double4*)a.tcen, (float4*)a.thalf);
    SSS_LAUNCH_CHECK(ctx, "k_tc_prep launch");
    const unsigned grid = (unsigned)(n_tblocks * n_chunks);
    void* args[] = {&a};
    SSS_CUDA_TRY(ctx, cudaLaunchKernel(kfn, dim3(grid), dim3(TC_NT), args, SMEM_BYTES, s));
    return SSS_OK;
}

}  // namespace sss_ap
