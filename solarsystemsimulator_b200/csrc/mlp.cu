// Learned short-range correction of the 3-D mesh force: a per-particle MLP
// 67 -> 128 -> 128 -> 3 (SiLU), bf16 weights and activations on the
// 5th-generation tensor cores (tcgen05.mma kind::f16, bf16 x bf16 -> f32 in
// tensor memory), trained online on the GPU by the kernels of this file.
//
// Layout: a CTA of 128 threads owns a tile of 128 rows (particles); thread
// r owns row r, which is TMEM lane r of every accumulator. Operands live in
// shared memory in the canonical no-swizzle K-major layout (core matrices of
// 8 rows x 16 bytes; K-adjacent core matrices 128 bytes apart, 8-row groups
// K * 16 bytes apart). One thread issues the MMAs (M = 128, K = 16 per
// instruction) and commits them to an mbarrier; every thread reads its own
// row of the result back with tcgen05.ld for the element-wise part (bias,
// SiLU, its derivative, bf16 rounding) and writes the next operand row.
//
// The weights reach shared memory as pre-built operand images (sss_mlp_pack
// writes them once per parameter update: W1^T, W2^T and W2 in the canonical
// layout, W3 row-major), one bulk async copy per CTA.
//
//   correction pass  k_mlp_correct_tc: inputs -> layer 1 -> layer 2 (tensor
//                    cores) -> 128 x 3 output layer (CUDA cores) -> KDK.
//   forward/backward k_mlp_rows_tc: the same forward, then the output delta,
//                    dZ2 = (dY W3^T) * silu'(Z2) (CUDA cores, K = 3),
//                    dH1 = dZ2 W2^T (tensor cores), dZ1 = dH1 * silu'(Z1);
//                    writes the activations and deltas the weight gradients
//                    need.
//   weight gradients k_mlp_tn_tc: dW = A^T dZ over the rows; the row tiles
//                    are transposed into K-major operands while staged
//                    (K = rows), the products accumulate in TMEM across the
//                    CTA's row tiles, and k_mlp_reduce adds the CTA partials
//                    in a fixed order, so gradients are deterministic.
//
// Rounding points: inputs, weights, hidden activations, output delta and
// hidden deltas are bf16; every sum is f32. The inputs are
// log1p(rho / rho_mean), evaluated once per mesh cell (k_mlp_lrho) and
// gathered per particle.

#include "pm3d.cuh"

#include <cuda_bf16.h>

#include <algorithm>

namespace {

constexpr int K1 = 80, HID = 128, K3 = 8;   // 67 inputs padded to 80
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + K1 * HID, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID;
constexpr int OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * K3, NPAR = OFF_B3 + K3;
static_assert(NPAR == SSS_MLP_N_PARAMS, "parameter layout");
static_assert(K1 == SSS_MLP_IN_PAD, "input width");

// operand images (bytes): W1^T (128 x 80), W2^T (128 x 128), W2 (128 x 128)
// in the canonical layout, W3 [128][8] row-major; all bf16
constexpr int IMG_W1T = 0;
constexpr int IMG_W2T = IMG_W1T + HID * K1 * 2;
constexpr int IMG_W2 = IMG_W2T + HID * HID * 2;
constexpr int IMG_W3 = IMG_W2 + HID * HID * 2;
constexpr int IMG_BYTES = IMG_W3 + HID * K3 * 2;
static_assert(IMG_BYTES == 4 * SSS_MLP_N_FRAGS, "operand image size");
static_assert(IMG_BYTES % 16 == 0 && IMG_W2T % 16 == 0 && IMG_W2 % 16 == 0 && IMG_W3 % 16 == 0, "bulk copies");

constexpr int ROWS = 128;   // rows per tile = threads per CTA = TMEM lanes

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x (low half) = lo
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

// SiLU and its derivative with the fast exponential and division (both a few
// ulp; the result is rounded to bf16 or multiplied into a bf16 delta)
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------- tcgen05 pieces
namespace tc {
// byte offset of element (r, k) of a canonical K-major bf16 operand with K columns
__device__ __forceinline__ int canon(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}
// shared-memory matrix descriptor: start, leading offset (K direction) 128 B,
// stride offset (8-row groups) K * 16 B, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t desc(uint32_t saddr, int K) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)((K * 16) >> 4) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// thread writes to shared memory -> visible to the tensor cores, all threads past
__device__ __forceinline__ void operands_ready() {
    fence_smem_to_async();
    fence_before();
    __syncthreads();
    fence_after();
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(tmem_d), "l"(da), "l"(db), "r"(id), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(sss_smem_addr(bar)) : "memory");
}
// D[tmem] = A[128 x K] B[N x K]^T over K / 16 instructions, then commit to bar
__device__ __forceinline__ void mma_layer(uint32_t tmem_d, uint32_t sa, uint32_t sb, int K, uint32_t id,
                                          uint64_t* bar) {
    for (int kk = 0; kk < K / 16; ++kk) mma(tmem_d, desc(sa + kk * 256, K), desc(sb + kk * 256, K), id, kk);
    commit(bar);
}

__device__ __forceinline__ void ld32(uint32_t addr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
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

// TMEM allocation by warp 0 (columns: a power of two >= 32)
__device__ __forceinline__ void alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(sss_smem_addr(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t tmem, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(cols) : "memory");
}
}  // namespace tc

// ---------------------------------------------------------------- packing

// One thread per bf16 element of the operand images.
__global__ void k_mlp_pack(const float* __restrict__ P, uint8_t* __restrict__ img) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    float w;
    int off;
    if (e < HID * K1) {                                  // W1^T: row = hidden unit n, K = input k
        const int n = e / K1, k = e % K1;
        w = P[OFF_W1 + k * HID + n];
        off = IMG_W1T + tc::canon(n, k, K1);
    } else if (e < HID * K1 + HID * HID) {               // W2^T: row = layer-2 unit n, K = layer-1 unit k
        const int l = e - HID * K1, n = l / HID, k = l % HID;
        w = P[OFF_W2 + k * HID + n];
        off = IMG_W2T + tc::canon(n, k, HID);
    } else if (e < HID * K1 + 2 * HID * HID) {           // W2: row = layer-1 unit i, K = layer-2 unit k
        const int l = e - HID * K1 - HID * HID, i = l / HID, k = l % HID;
        w = P[OFF_W2 + i * HID + k];
        off = IMG_W2 + tc::canon(i, k, HID);
    } else if (e < HID * K1 + 2 * HID * HID + HID * K3) {  // W3 row-major
        const int l = e - HID * K1 - 2 * HID * HID;
        w = P[OFF_W3 + l];
        off = IMG_W3 + 2 * l;
    } else {
        return;
    }
    *reinterpret_cast<__nv_bfloat16*>(img + off) = __float2bfloat16_rn(w);
}

// ------------------------------------------------------------- features

// lrho[c] = log1p(rho[c] * inv_mean) for every mesh cell
__global__ void k_mlp_lrho(const float* __restrict__ rho, long long n3, float inv_mean, float* __restrict__ out) {
    const long long i0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (i0 + 3 < n3) {
        const float4 v = *reinterpret_cast<const float4*>(rho + i0);
        *reinterpret_cast<float4*>(out + i0) =
            make_float4(log1pf(v.x * inv_mean), log1pf(v.y * inv_mean), log1pf(v.z * inv_mean),
                        log1pf(v.w * inv_mean));
    } else {
        for (long long i = i0; i < n3; ++i) out[i] = log1pf(rho[i] * inv_mean);
    }
}

// The 40 bf16 pairs of the input row of particle p (p < 0: zeros): the 4x4x4
// cells (i0-1 .. i0+2 per axis, wrapped) of the log-density mesh, then the
// sub-cell offsets t - 1/2, then zeros.
__device__ __forceinline__ void feature_row(const Pm3Parts& s, const float* __restrict__ lrho, int n,
                                            double inv_h, long long p, uint32_t (&row)[K1 / 2]) {
#pragma unroll
    for (int q = 0; q < K1 / 2; ++q) row[q] = 0u;
    if (p < 0) return;
    int i[3];
    double t[3];
    for (int c = 0; c < 3; ++c) pm3_cell(s.x[c][p], inv_h, n, i[c], t[c]);
    long long ox[4];
    int oy[4], oz[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int ix = i[0] + a - 1, iy = i[1] + a - 1, iz = i[2] + a - 1;
        ix += ix < 0 ? n : 0;
        ix -= ix >= n ? n : 0;
        iy += iy < 0 ? n : 0;
        iy -= iy >= n ? n : 0;
        iz += iz < 0 ? n : 0;
        iz -= iz >= n ? n : 0;
        ox[a] = (long long)ix * n * n;
        oy[a] = iy * n;
        oz[a] = iz;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; c += 2)
                row[a * 8 + b * 2 + c / 2] =
                    pack2(__ldg(lrho + ox[a] + oy[b] + oz[c]), __ldg(lrho + ox[a] + oy[b] + oz[c + 1]));
    row[32] = pack2((float)(t[0] - 0.5), (float)(t[1] - 0.5));
    row[33] = pack2((float)(t[2] - 0.5), 0.0f);
}

// features of selected particles (sss_mlp_features): one row per thread
__global__ void k_mlp_features(const Pm3Parts s, const float* __restrict__ lrho, int n, double inv_h,
                               const long long* __restrict__ idx, long long rows, uint16_t* __restrict__ X) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    long long p = idx ? idx[r] : r;
    if (p >= s.n || p < 0) p = -1;
    uint32_t row[K1 / 2];
    feature_row(s, lrho, n, inv_h, p, row);
    uint4* dst = reinterpret_cast<uint4*>(X + r * K1);
#pragma unroll
    for (int j = 0; j < K1 / 8; ++j) dst[j] = make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
}

// row r of a canonical K1-wide operand tile from 40 bf16 pairs
__device__ __forceinline__ void put_row80(uint8_t* tile, int r, const uint32_t (&row)[K1 / 2]) {
#pragma unroll
    for (int j = 0; j < K1 / 8; ++j)
        *reinterpret_cast<uint4*>(tile + tc::canon(r, 8 * j, K1)) =
            make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
}

// ------------------------------------------------- shared-memory plans
// correction pass (2 CTAs per SM): W1^T | W2^T | W3 | X tile (128 x 80) |
// H tile (128 x 128) | f32 b1[128] b2[128] b3[8] W3[128][3] | barriers, TMEM slot
// forward/backward: W1^T | W2^T | W2 | W3 | X | H | D tile (128 x 128) | f32 | barriers
struct Plan {
    int w1t, w2t, w2, w3, x, h, d, f, bar, bytes;
};
constexpr int N_F = HID + HID + K3 + HID * 3;
constexpr Plan plan_of(bool full) {
    const int w3 = full ? IMG_W3 : IMG_W2;
    const int x = w3 + HID * K3 * 2;
    const int h = x + ROWS * K1 * 2;
    const int d = full ? h + ROWS * HID * 2 : -1;
    const int f = (full ? d : h) + ROWS * HID * 2;
    const int bar = (f + N_F * 4 + 15) / 16 * 16;
    return Plan{IMG_W1T, IMG_W2T, full ? IMG_W2 : -1, w3, x, h, d, f, bar, bar + 32};
}
constexpr Plan PLAN_C = plan_of(false);
constexpr Plan PLAN_R = plan_of(true);
static_assert(2 * PLAN_C.bytes <= 227 * 1024, "two correction CTAs per SM");
static_assert(PLAN_R.bytes <= 227 * 1024, "shared memory of the training kernel");
constexpr uint32_t TMEM_COLS = 256;   // layer 1 | layer 2 (the backward reuses layer 2's columns)

struct SmemView {
    uint8_t* base;
    Plan pl;
    float* b1;
    float* b2;
    float* b3;
    float* w3;       // [128][3] f32 of the bf16 weights
    uint64_t* bar;   // [0] images, [1] MMAs
    uint32_t* tslot;
};

// Barriers, TMEM, biases; the images by bulk copies (FULL: all four, else
// W1^T, W2^T and W3); W3 widened to f32. Returns false (status set) if the
// copies did not arrive in time.
template <bool FULL>
__device__ __forceinline__ bool stage_weights(SmemView& v, uint8_t* base, const float* __restrict__ P,
                                              const uint8_t* __restrict__ img, int* status) {
    const int tid = threadIdx.x;
    v.base = base;
    v.pl = FULL ? PLAN_R : PLAN_C;
    v.b1 = reinterpret_cast<float*>(base + v.pl.f);
    v.b2 = v.b1 + HID;
    v.b3 = v.b2 + HID;
    v.w3 = v.b3 + K3;
    v.bar = reinterpret_cast<uint64_t*>(base + v.pl.bar);
    v.tslot = reinterpret_cast<uint32_t*>(base + v.pl.bar + 16);
    if (tid == 0) {
        sss_mbar_init(&v.bar[0], 1);
        sss_mbar_init(&v.bar[1], 1);
        sss_fence_mbar_init();
    }
    if ((tid >> 5) == 0) tc::alloc(v.tslot, TMEM_COLS);
    for (int i = tid; i < HID; i += blockDim.x) {
        v.b1[i] = P[OFF_B1 + i];
        v.b2[i] = P[OFF_B2 + i];
    }
    if (tid < K3) v.b3[tid] = P[OFF_B3 + tid];
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (tid == 0) {
        if (FULL) {
            sss_mbar_arrive_expect_tx(&v.bar[0], IMG_BYTES);
            sss_bulk_g2s(base, img, IMG_BYTES, &v.bar[0]);
        } else {
            sss_mbar_arrive_expect_tx(&v.bar[0], IMG_W2 + HID * K3 * 2);
            sss_bulk_g2s(base, img, IMG_W2, &v.bar[0]);
            sss_bulk_g2s(base + v.pl.w3, img + IMG_W3, HID * K3 * 2, &v.bar[0]);
        }
    }
    const bool ok = sss_mbar_wait_bounded(&v.bar[0], 0, status);
    if (ok) {
        const uint16_t* w3 = reinterpret_cast<const uint16_t*>(base + v.pl.w3);
        for (int i = tid; i < HID * 3; i += blockDim.x)
            v.w3[i] = __uint_as_float((uint32_t)w3[(i / 3) * K3 + i % 3] << 16);
    }
    return !__syncthreads_or(!ok);
}

__device__ __forceinline__ void release_tmem(const SmemView& v) {
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if ((threadIdx.x >> 5) == 0) tc::dealloc(*v.tslot, TMEM_COLS);
}

// Layer 1 (X tile already staged): Z1 -> d1; H1 = bf16(silu(Z1 + b1)) into
// the H tile and, when h1_out is given, into h1_out (64 bf16 pairs).
// Layer 2: Z2 -> d2. Returns false on a timed-out wait.
__device__ __forceinline__ bool hidden_layers(const SmemView& v, uint32_t d1, uint32_t d2, unsigned& phase,
                                              int* status, uint32_t* h1_out) {
    const int tid = threadIdx.x;
    const uint32_t lane_base = (uint32_t)(32 * (tid >> 5)) << 16;
    tc::operands_ready();
    if (tid == 0)
        tc::mma_layer(d1, sss_smem_addr(v.base + v.pl.x), sss_smem_addr(v.base + v.pl.w1t), K1,
                      tc::idesc(HID), &v.bar[1]);
    bool bad = !sss_mbar_wait_bounded(&v.bar[1], phase, status);
    phase ^= 1u;
    if (__syncthreads_or(bad)) return false;
    tc::fence_after();
#pragma unroll 1
    for (int j2 = 0; j2 < HID / 32; ++j2) {
        float z[32];
        tc::ld32(d1 + lane_base + 32 * j2, z);
        tc::wait_ld();
        uint32_t h[16];
#pragma unroll
        for (int q = 0; q < 16; ++q)
            h[q] = pack2(silu(z[2 * q] + v.b1[32 * j2 + 2 * q]), silu(z[2 * q + 1] + v.b1[32 * j2 + 2 * q + 1]));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint4 w = make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
            *reinterpret_cast<uint4*>(v.base + v.pl.h + tc::canon(tid, 32 * j2 + 8 * u, HID)) = w;
            if (h1_out) reinterpret_cast<uint4*>(h1_out)[4 * j2 + u] = w;
        }
    }
    tc::operands_ready();
    if (tid == 0)
        tc::mma_layer(d2, sss_smem_addr(v.base + v.pl.h), sss_smem_addr(v.base + v.pl.w2t), HID,
                      tc::idesc(HID), &v.bar[1]);
    bad = !sss_mbar_wait_bounded(&v.bar[1], phase, status);
    phase ^= 1u;
    if (__syncthreads_or(bad)) return false;
    tc::fence_after();
    return true;
}

// Layer 2's activations and the 128 x 3 output layer on the CUDA cores:
// y = b3 + bf16(silu(Z2 + b2)) W3; h2_out (nullable) receives the bf16 row.
__device__ __forceinline__ void output_layer(const SmemView& v, uint32_t d2, float& y0, float& y1, float& y2,
                                             uint32_t* h2_out) {
    const uint32_t lane_base = (uint32_t)(32 * (threadIdx.x >> 5)) << 16;
    y0 = v.b3[0];
    y1 = v.b3[1];
    y2 = v.b3[2];
#pragma unroll 1
    for (int j2 = 0; j2 < HID / 32; ++j2) {
        float z[32];
        tc::ld32(d2 + lane_base + 32 * j2, z);
        tc::wait_ld();
        uint32_t h[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int k = 32 * j2 + 2 * q;
            h[q] = pack2(silu(z[2 * q] + v.b2[k]), silu(z[2 * q + 1] + v.b2[k + 1]));
            const float ha = bf_lo(h[q]), hb = bf_hi(h[q]);
            y0 = fmaf(ha, v.w3[3 * k], y0);
            y1 = fmaf(ha, v.w3[3 * k + 1], y1);
            y2 = fmaf(ha, v.w3[3 * k + 2], y2);
            y0 = fmaf(hb, v.w3[3 * k + 3], y0);
            y1 = fmaf(hb, v.w3[3 * k + 4], y1);
            y2 = fmaf(hb, v.w3[3 * k + 5], y2);
        }
        if (h2_out)
#pragma unroll
            for (int u = 0; u < 4; ++u)
                reinterpret_cast<uint4*>(h2_out)[4 * j2 + u] =
                    make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
    }
}

// ------------------------------------------------------- correction pass

__global__ void __launch_bounds__(ROWS, 2) k_mlp_correct_tc(const Pm3Parts s, const float* __restrict__ lrho,
                                                            int n, double inv_h, const float* __restrict__ P,
                                                            const uint8_t* __restrict__ img, double out_scale,
                                                            const Pm3Epi e, int* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    SmemView v;
    const int tid = threadIdx.x;
    const bool ok = stage_weights<false>(v, smem, P, img, status);
    const uint32_t tmem = *v.tslot, d1 = tmem, d2 = tmem + HID;
    unsigned phase = 0;
    const long long tiles = (s.n + ROWS - 1) / ROWS;
    uint32_t row[K1 / 2];
    if (ok && blockIdx.x < tiles) {
        const long long p = (long long)blockIdx.x * ROWS + tid;
        feature_row(s, lrho, n, inv_h, p < s.n ? p : -1, row);
        put_row80(smem + v.pl.x, tid, row);
    }
    for (long long tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x) {
        const long long p = tile * ROWS + tid;
        tc::operands_ready();
        if (tid == 0)
            tc::mma_layer(d1, sss_smem_addr(smem + v.pl.x), sss_smem_addr(smem + v.pl.w1t), K1,
                          tc::idesc(HID), &v.bar[1]);
        bool bad = !sss_mbar_wait_bounded(&v.bar[1], phase, status);
        phase ^= 1u;
        if (__syncthreads_or(bad)) break;
        tc::fence_after();
        const uint32_t lane_base = (uint32_t)(32 * (tid >> 5)) << 16;
#pragma unroll 1
        for (int j2 = 0; j2 < HID / 32; ++j2) {
            float z[32];
            tc::ld32(d1 + lane_base + 32 * j2, z);
            tc::wait_ld();
            uint32_t h[16];
#pragma unroll
            for (int q = 0; q < 16; ++q)
                h[q] = pack2(silu(z[2 * q] + v.b1[32 * j2 + 2 * q]), silu(z[2 * q + 1] + v.b1[32 * j2 + 2 * q + 1]));
#pragma unroll
            for (int u = 0; u < 4; ++u)
                *reinterpret_cast<uint4*>(smem + v.pl.h + tc::canon(tid, 32 * j2 + 8 * u, HID)) =
                    make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
        }
        tc::operands_ready();
        if (tid == 0)
            tc::mma_layer(d2, sss_smem_addr(smem + v.pl.h), sss_smem_addr(smem + v.pl.w2t), HID,
                          tc::idesc(HID), &v.bar[1]);
        // the X tile is free once layer 1 has completed: gather the next
        // tile's inputs while layer 2 runs
        if (tile + gridDim.x < tiles) {
            const long long pn = (tile + gridDim.x) * ROWS + tid;
            feature_row(s, lrho, n, inv_h, pn < s.n ? pn : -1, row);
            put_row80(smem + v.pl.x, tid, row);
        }
        bad = !sss_mbar_wait_bounded(&v.bar[1], phase, status);
        phase ^= 1u;
        if (__syncthreads_or(bad)) break;
        tc::fence_after();
        float y0, y1, y2;
        output_layer(v, d2, y0, y1, y2, nullptr);
        if (p < s.n) {
            const double ax = s.a[0][p] + out_scale * (double)y0;
            const double ay = s.a[1][p] + out_scale * (double)y1;
            const double az = s.a[2][p] + out_scale * (double)y2;
            pm3_epilogue(s, e, p, ax, ay, az);
        }
    }
    release_tmem(v);
}

// ------------------------------------------------- forward and backward

struct RowBufs {
    uint32_t* Xc;       // [rows_pad][40] compacted inputs (when idx is given)
    uint32_t* H1;       // [rows_pad][64] bf16 pairs
    uint32_t* H2;
    uint32_t* dZ1;
    uint32_t* dZ2;
    uint32_t* dY;       // [rows_pad][4]: 8 bf16, columns 3..7 zero
    float* loss;        // [gridDim.x] per-CTA sums of squared errors
};

// TRAIN = false: forward only, Y[r][0..3) <- outputs of rows r < rows.
// TRAIN = true: forward and backward of rows idx[r] (idx NULL: r) of X, T.
template <bool TRAIN>
__global__ void __launch_bounds__(ROWS, 1) k_mlp_rows_tc(const uint16_t* __restrict__ X,
                                                         const float* __restrict__ T, const int* __restrict__ idx,
                                                         long long rows, long long x_rows, long long rows_pad,
                                                         float dscale, const float* __restrict__ P,
                                                         const uint8_t* __restrict__ img, const RowBufs B,
                                                         float* __restrict__ Y, int* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    SmemView v;
    const int tid = threadIdx.x;
    const bool ok = stage_weights<true>(v, smem, P, img, status);
    const uint32_t tmem = *v.tslot, d1 = tmem, d2 = tmem + HID;
    const uint32_t lane_base = (uint32_t)(32 * (tid >> 5)) << 16;
    unsigned phase = 0;
    float lsum = 0.0f;
    const long long tiles = rows_pad / ROWS;
    for (long long tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x) {
        const long long r = tile * ROWS + tid;
        long long sr = -1;                        // source row of X and T
        if (r < rows) {
            sr = idx ? (long long)idx[r] : r;
            if (sr >= x_rows || sr < 0) sr = -1;  // an index outside X reads as a zero row with no target
        }
        // ---- inputs
        uint32_t row[K1 / 2];
        if (sr >= 0) {
            const uint4* src = reinterpret_cast<const uint4*>(X + sr * K1);
#pragma unroll
            for (int j = 0; j < K1 / 8; ++j) {
                const uint4 w = src[j];
                row[4 * j] = w.x; row[4 * j + 1] = w.y; row[4 * j + 2] = w.z; row[4 * j + 3] = w.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < K1 / 2; ++q) row[q] = 0u;
        }
        put_row80(smem + v.pl.x, tid, row);
        if (TRAIN && B.Xc)
#pragma unroll
            for (int j = 0; j < K1 / 8; ++j)
                reinterpret_cast<uint4*>(B.Xc + r * (K1 / 2))[j] =
                    make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
        // ---- layers 1 and 2 on the tensor cores
        if (!hidden_layers(v, d1, d2, phase, status, TRAIN ? B.H1 + r * (HID / 2) : nullptr)) break;
        float y0, y1, y2;
        output_layer(v, d2, y0, y1, y2, TRAIN ? B.H2 + r * (HID / 2) : nullptr);
        if (!TRAIN) {
            if (r < rows) {
                Y[r * 3] = y0;
                Y[r * 3 + 1] = y1;
                Y[r * 3 + 2] = y2;
            }
            continue;
        }
        // ---- output delta dY = dscale (Y - T), bf16
        float dl0 = 0.0f, dl1 = 0.0f, dl2 = 0.0f;
        if (sr >= 0) {
            const float e0 = y0 - T[sr * 3], e1 = y1 - T[sr * 3 + 1], e2 = y2 - T[sr * 3 + 2];
            dl0 = dscale * e0;
            dl1 = dscale * e1;
            dl2 = dscale * e2;
            lsum += e0 * e0 + e1 * e1 + e2 * e2;
        }
        const uint32_t a01 = pack2(dl0, dl1), a2 = pack2(dl2, 0.0f);
        reinterpret_cast<uint4*>(B.dY)[r] = make_uint4(a01, a2, 0u, 0u);
        const float g0 = bf_lo(a01), g1 = bf_hi(a01), g2 = bf_lo(a2);
        // ---- dZ2 = bf16((dY W3^T) * silu'(Z2 + b2)) into the D tile (K-major, K = layer-2 units)
#pragma unroll 1
        for (int j2 = 0; j2 < HID / 32; ++j2) {
            float z[32];
            tc::ld32(d2 + lane_base + 32 * j2, z);
            tc::wait_ld();
            uint32_t h[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                float dz[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int k = 32 * j2 + 2 * q + u;
                    float dh = g0 * v.w3[3 * k];
                    dh = fmaf(g1, v.w3[3 * k + 1], dh);
                    dh = fmaf(g2, v.w3[3 * k + 2], dh);
                    dz[u] = dh * dsilu(z[2 * q + u] + v.b2[k]);
                }
                h[q] = pack2(dz[0], dz[1]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint4 w = make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
                *reinterpret_cast<uint4*>(smem + v.pl.d + tc::canon(tid, 32 * j2 + 8 * u, HID)) = w;
                reinterpret_cast<uint4*>(B.dZ2 + r * (HID / 2))[4 * j2 + u] = w;
            }
        }
        // ---- dH1 = dZ2 W2^T on the tensor cores (into layer 2's columns)
        tc::operands_ready();
        if (tid == 0)
            tc::mma_layer(d2, sss_smem_addr(smem + v.pl.d), sss_smem_addr(smem + v.pl.w2), HID,
                          tc::idesc(HID), &v.bar[1]);
        const bool bad = !sss_mbar_wait_bounded(&v.bar[1], phase, status);
        phase ^= 1u;
        if (__syncthreads_or(bad)) break;
        tc::fence_after();
        // ---- dZ1 = bf16(dH1 * silu'(Z1 + b1))
#pragma unroll 1
        for (int j2 = 0; j2 < HID / 32; ++j2) {
            float dh[32], z[32];
            tc::ld32(d2 + lane_base + 32 * j2, dh);
            tc::ld32(d1 + lane_base + 32 * j2, z);
            tc::wait_ld();
            uint32_t h[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int k = 32 * j2 + 2 * q;
                h[q] = pack2(dh[2 * q] * dsilu(z[2 * q] + v.b1[k]), dh[2 * q + 1] * dsilu(z[2 * q + 1] + v.b1[k + 1]));
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                reinterpret_cast<uint4*>(B.dZ1 + r * (HID / 2))[4 * j2 + u] =
                    make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
        }
    }
    if (TRAIN) {
        // the CTA's sum of squared errors (fixed order: warps, then lanes by shuffles)
        __shared__ float red[ROWS / 32];
#pragma unroll
        for (int off = 16; off; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
        if ((tid & 31) == 0) red[tid >> 5] = lsum;
        __syncthreads();
        if (tid == 0) B.loss[blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
    }
    release_tmem(v);
}

// ------------------------------------------------------ weight gradients

// D[m][n] = sum over rows r of Pm[r][m] Qm[r][n] (Pm: 128 bf16 columns, row
// stride ldp; Qm: nq of NQ columns, row stride ldq) over the CTA's rows
// [blockIdx.x * per, +per) of S, on the tensor cores. Row tiles of 128 are
// transposed while staged into K-major operands (K = rows; rows beyond S
// read as zeros). part[c] receives D (transposed ? part[n * 128 + m] :
// part[m * nq + n]) and then the column sums of Pm (sum_p) or of Qm.
namespace tn {
constexpr int OFF_P = 0;                      // 128 x 128 bf16 canonical
constexpr int OFF_Q = OFF_P + 128 * ROWS * 2; // NQ x 128
constexpr int OFF_BAR = OFF_Q + 128 * ROWS * 2;
constexpr int BYTES = OFF_BAR + 16;
}  // namespace tn

// rows [b, b + 128) of a bf16 matrix (ncol columns, of which nreal carry data)
// transposed into a canonical operand (row = column of the matrix, K = row)
__device__ __forceinline__ void stage_transposed(const uint16_t* __restrict__ M, int ld, int ncol, int nreal,
                                                 long long b, long long S, uint8_t* tile) {
    const int pairs = ncol / 2;
    for (int it = threadIdx.x; it < pairs * (ROWS / 8); it += blockDim.x) {
        const int cp = it % pairs, g = it / pairs;
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const long long row = b + 8 * g + q;
            w[q] = (row < S && 2 * cp < nreal) ? *reinterpret_cast<const uint32_t*>(M + row * ld + 2 * cp) : 0u;
        }
        const uint4 lo = make_uint4((w[0] & 0xffffu) | (w[1] << 16), (w[2] & 0xffffu) | (w[3] << 16),
                                    (w[4] & 0xffffu) | (w[5] << 16), (w[6] & 0xffffu) | (w[7] << 16));
        const uint4 hi = make_uint4((w[0] >> 16) | (w[1] & 0xffff0000u), (w[2] >> 16) | (w[3] & 0xffff0000u),
                                    (w[4] >> 16) | (w[5] & 0xffff0000u), (w[6] >> 16) | (w[7] & 0xffff0000u));
        *reinterpret_cast<uint4*>(tile + tc::canon(2 * cp, 8 * g, ROWS)) = lo;
        *reinterpret_cast<uint4*>(tile + tc::canon(2 * cp + 1, 8 * g, ROWS)) = hi;
    }
}

// sum over the 128 rows (K) of row c of a staged canonical operand, ascending
__device__ __forceinline__ float staged_row_sum(const uint8_t* tile, int c) {
    float s = 0.0f;
#pragma unroll 4
    for (int k8 = 0; k8 < ROWS / 8; ++k8) {
        const uint4 w = *reinterpret_cast<const uint4*>(tile + tc::canon(c, 8 * k8, ROWS));
        const uint32_t q[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            s += bf_lo(q[u]);
            s += bf_hi(q[u]);
        }
    }
    return s;
}

template <int NQ>
__global__ void __launch_bounds__(ROWS, 1) k_mlp_tn_tc(const uint16_t* __restrict__ Pm, int ldp,
                                                       const uint16_t* __restrict__ Qm, int ldq, int nq, long long S,
                                                       long long per, int transposed, int sum_p,
                                                       float* __restrict__ part, int* status) {
    constexpr uint32_t COLS = NQ <= 32 ? 32 : (NQ <= 64 ? 64 : 128);
    static_assert(NQ % 16 == 0 && NQ >= 16 && NQ <= 128, "N of the gradient MMA");
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + tn::OFF_BAR);
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x;
    if (tid == 0) {
        sss_mbar_init(bar, 1);
        sss_fence_mbar_init();
    }
    if ((tid >> 5) == 0) tc::alloc(&tslot, COLS);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t d = tslot;
    const long long r0 = (long long)blockIdx.x * per;
    const long long r1 = min(S, r0 + per);
    const int nsum = sum_p ? 128 : nq;
    float cs = 0.0f;
    unsigned phase = 0;
    bool any = false, bad = false;
    for (long long b = r0; b < r1; b += ROWS) {
        stage_transposed(Pm, ldp, 128, 128, b, r1, smem + tn::OFF_P);
        stage_transposed(Qm, ldq, NQ, nq, b, r1, smem + tn::OFF_Q);
        tc::operands_ready();
        if (tid < nsum) cs += staged_row_sum(smem + (sum_p ? tn::OFF_P : tn::OFF_Q), tid);
        if (tid == 0) {
            const uint32_t sp = sss_smem_addr(smem + tn::OFF_P), sq = sss_smem_addr(smem + tn::OFF_Q);
            for (int kk = 0; kk < ROWS / 16; ++kk)
                tc::mma(d, tc::desc(sp + kk * 256, ROWS), tc::desc(sq + kk * 256, ROWS), tc::idesc(NQ),
                        (any || kk > 0) ? 1 : 0);
            tc::commit(bar);
        }
        bad = !sss_mbar_wait_bounded(bar, phase, status);
        phase ^= 1u;
        if (__syncthreads_or(bad)) break;
        tc::fence_after();
        any = true;
    }
    float* out = part + (long long)blockIdx.x * (128 * nq + nsum);
    if (!bad) {
        const uint32_t lane_base = (uint32_t)(32 * (tid >> 5)) << 16;
#pragma unroll 1
        for (int c0 = 0; c0 < NQ; c0 += 16) {
            float v[16];
            if (any) {
                tc::ld16(d + lane_base + c0, v);
                tc::wait_ld();
            } else {
#pragma unroll
                for (int q = 0; q < 16; ++q) v[q] = 0.0f;
            }
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int c = c0 + q;
                if (c < nq) {
                    if (transposed) out[c * 128 + tid] = v[q];
                    else out[tid * nq + c] = v[q];
                }
            }
        }
        if (tid < nsum) out[128 * nq + tid] = cs;
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if ((tid >> 5) == 0) tc::dealloc(d, COLS);
}

__global__ void k_mlp_reduce(const float* __restrict__ part, int ctas, int MN, int N, float* __restrict__ gW,
                             float* __restrict__ gb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MN + N) return;
    float s = 0.0f;
    for (int c = 0; c < ctas; ++c) s += part[(long long)c * (MN + N) + i];
    if (i < MN) gW[i] = s;
    else gb[i - MN] = s;
}

__global__ void k_mlp_loss(const float* __restrict__ part, long long cnt, float scale, float* __restrict__ loss) {
    float s = 0.0f;
    for (long long i = threadIdx.x; i < cnt; i += blockDim.x) s += part[i];
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] * scale;
}

__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m,
                           float* __restrict__ v, long long n, float lr_t, float b1, float b2, float eps_t) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gr[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps_t);
}

// one weight gradient: S rows split into CTAs of whole 128-row tiles
int tn_gemm(sss_ctx* ctx, const uint16_t* Pm, int ldp, const uint16_t* Qm, int ldq, int nq, long long S,
            int transposed, int sum_p, float* part, float* gW, float* gb, cudaStream_t st) {
    const long long tiles = std::max<long long>(1, (S + ROWS - 1) / ROWS);
    const long long per_t = (tiles + ctx->num_sms - 1) / ctx->num_sms;
    const long long per = per_t * ROWS;
    const int ctas = (int)((tiles + per_t - 1) / per_t);
    const int smem = tn::BYTES;
    if (nq > 16) {
        SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_tn_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_tn_tc<80>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        if (nq == 80)
            k_mlp_tn_tc<80><<<ctas, ROWS, smem, st>>>(Pm, ldp, Qm, ldq, nq, S, per, transposed, sum_p, part,
                                                      ctx->d_status);
        else
            k_mlp_tn_tc<128><<<ctas, ROWS, smem, st>>>(Pm, ldp, Qm, ldq, nq, S, per, transposed, sum_p, part,
                                                       ctx->d_status);
    } else {
        SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_tn_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_mlp_tn_tc<16><<<ctas, ROWS, smem, st>>>(Pm, ldp, Qm, ldq, nq, S, per, transposed, sum_p, part,
                                                  ctx->d_status);
    }
    SSS_LAUNCH_CHECK(ctx, "k_mlp_tn_tc");
    const int nsum = sum_p ? 128 : nq;
    const int tot = 128 * nq + nsum;
    k_mlp_reduce<<<(tot + 255) / 256, 256, 0, st>>>(part, ctas, 128 * nq, nsum, gW, gb);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_reduce");
    return SSS_OK;
}

// log1p(rho / rho_mean) of every cell of the plan's mesh into p->lrho
int log_density(sss_ctx* ctx, sss_pm3* p, double rho_mean, cudaStream_t st) {
    const long long n3 = (long long)p->n * p->n * p->n;
    const long long quads = (n3 + 3) / 4;
    k_mlp_lrho<<<(unsigned)((quads + 255) / 256), 256, 0, st>>>(p->rho, n3, (float)(1.0 / rho_mean), p->lrho);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_lrho");
    return SSS_OK;
}

}  // namespace

extern "C" int sss_mlp_pack(sss_ctx* ctx, const float* params, uint32_t* frags, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!params || !frags) return sss_set_err(ctx, SSS_ERR_ARG, "NULL parameters or operand images");
    const int elems = IMG_BYTES / 2;
    k_mlp_pack<<<(elems + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, reinterpret_cast<uint8_t*>(frags));
    SSS_LAUNCH_CHECK(ctx, "k_mlp_pack");
    return SSS_OK;
}

extern "C" int sss_mlp_features(sss_ctx* ctx, sss_pm3* p, const sss_pm3_particles* s, const int64_t* idx,
                                int64_t rows, double rho_mean, uint16_t* X, void* stream) {
    if (!ctx || !p || !s) return SSS_ERR_ARG;
    if (rows < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative row count");
    if (rows == 0) return SSS_OK;
    if (!X || !s->x[0] || !s->x[1] || !s->x[2]) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    if (!(rho_mean > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "rho_mean must be > 0");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = log_density(ctx, p, rho_mean, st);
    if (rc) return rc;
    const unsigned blocks = (unsigned)((rows + 127) / 128);
    k_mlp_features<<<blocks, 128, 0, st>>>(pm3_parts(s), p->lrho, p->n, p->n / p->box, (const long long*)idx, rows,
                                           X);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_features");
    return SSS_OK;
}

extern "C" int sss_mlp_forward(sss_ctx* ctx, const float* params, const uint32_t* frags, const uint16_t* X,
                               int64_t rows, float* Y, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (rows < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative row count");
    if (rows == 0) return SSS_OK;
    if (!params || !frags || !X || !Y) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_rows_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           PLAN_R.bytes));
    const long long rows_pad = (rows + ROWS - 1) / ROWS * ROWS;
    const int blocks = (int)std::min<long long>(rows_pad / ROWS, (long long)ctx->num_sms);
    RowBufs B{};
    k_mlp_rows_tc<false><<<blocks, ROWS, PLAN_R.bytes, (cudaStream_t)stream>>>(
        X, nullptr, nullptr, rows, rows, rows_pad, 0.0f, params, reinterpret_cast<const uint8_t*>(frags), B, Y,
        ctx->d_status);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_rows_tc (forward)");
    return SSS_OK;
}

extern "C" int sss_mlp_correct(sss_ctx* ctx, sss_pm3* p, const sss_pm3_particles* s, const float* params,
                               const uint32_t* frags, double rho_mean, double out_scale, int mode, double hdt,
                               double dt, float* snap, void* stream) {
    if (!ctx || !p || !s) return SSS_ERR_ARG;
    if (s->n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative particle count");
    if (s->n == 0) return SSS_OK;
    if (!params || !frags) return sss_set_err(ctx, SSS_ERR_ARG, "NULL parameters or operand images");
    for (int c = 0; c < 3; ++c)
        if (!s->x[c] || !s->v[c] || !s->a[c]) return sss_set_err(ctx, SSS_ERR_ARG, "NULL particle array");
    if (!(rho_mean > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "rho_mean must be > 0");
    if (mode < SSS_PM3_FORCE || mode > SSS_PM3_KICK_DRIFT) return sss_set_err(ctx, SSS_ERR_ARG, "bad mode");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = log_density(ctx, p, rho_mean, st);
    if (rc) return rc;
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_correct_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, PLAN_C.bytes));
    const long long tiles = (s->n + ROWS - 1) / ROWS;
    const int blocks = (int)std::min<long long>(tiles, (long long)ctx->num_sms * 2);
    Pm3Epi e{mode, hdt, dt, p->box, snap};
    k_mlp_correct_tc<<<blocks, ROWS, PLAN_C.bytes, st>>>(pm3_parts(s), p->lrho, p->n, p->n / p->box, params,
                                                      reinterpret_cast<const uint8_t*>(frags), out_scale, e,
                                                      ctx->d_status);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_correct");
    return SSS_OK;
}

extern "C" int sss_mlp_grad(sss_ctx* ctx, const float* params, const uint32_t* frags, const uint16_t* X,
                            const float* T, int64_t x_rows, const int32_t* idx, int64_t rows, float* grads,
                            float* loss, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (rows < 1) return sss_set_err(ctx, SSS_ERR_ARG, "need at least one row");
    if (x_rows < (idx ? 1 : rows)) return sss_set_err(ctx, SSS_ERR_ARG, "X holds fewer rows than selected");
    if (!params || !frags || !X || !T || !grads) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    cudaStream_t st = (cudaStream_t)stream;
    const long long rows_pad = (rows + ROWS - 1) / ROWS * ROWS;
    const int blocks = (int)std::min<long long>(rows_pad / ROWS, (long long)ctx->num_sms);
    // scratch: row buffers, loss partials, GEMM partials
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t oXc = take(idx ? (size_t)rows_pad * K1 * 2 : 0);
    const size_t oH1 = take((size_t)rows_pad * HID * 2), oH2 = take((size_t)rows_pad * HID * 2);
    const size_t oZ1 = take((size_t)rows_pad * HID * 2), oZ2 = take((size_t)rows_pad * HID * 2);
    const size_t oY = take((size_t)rows_pad * K3 * 2);
    const size_t oL = take((size_t)blocks * 4);
    const size_t oP = take((size_t)ctx->num_sms * (HID * HID + HID) * 4);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* base = (char*)scr;
    RowBufs B;
    B.Xc = idx ? (uint32_t*)(base + oXc) : nullptr;
    B.H1 = (uint32_t*)(base + oH1);
    B.H2 = (uint32_t*)(base + oH2);
    B.dZ1 = (uint32_t*)(base + oZ1);
    B.dZ2 = (uint32_t*)(base + oZ2);
    B.dY = (uint32_t*)(base + oY);
    B.loss = (float*)(base + oL);
    float* part = (float*)(base + oP);
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_rows_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           PLAN_R.bytes));
    const float dscale = (float)(2.0 / (3.0 * (double)rows));
    k_mlp_rows_tc<true><<<blocks, ROWS, PLAN_R.bytes, st>>>(X, T, idx, rows, x_rows, rows_pad, dscale, params,
                                                        reinterpret_cast<const uint8_t*>(frags), B, nullptr,
                                                        ctx->d_status);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_rows_tc");
    const uint16_t* Xg = idx ? (const uint16_t*)B.Xc : X;
    // X rows beyond `rows` are read only when idx is NULL; pad rows of the
    // deltas are zero, so those products vanish, but the reads must stay in
    // the caller's array: use S = rows there
    const long long S1 = idx ? rows_pad : rows;
    // dW1^T = dZ1^T X (written transposed into W1[in][out]); b1 = column sums of dZ1
    rc = tn_gemm(ctx, (const uint16_t*)B.dZ1, HID, Xg, K1, K1, S1, 1, 1, part, grads + OFF_W1, grads + OFF_B1, st);
    if (rc) return rc;
    // dW2 = H1^T dZ2; b2 = column sums of dZ2
    rc = tn_gemm(ctx, (const uint16_t*)B.H1, HID, (const uint16_t*)B.dZ2, HID, HID, rows_pad, 0, 0, part,
                 grads + OFF_W2, grads + OFF_B2, st);
    if (rc) return rc;
    // dW3 = H2^T dY (8 columns); b3 = column sums of dY
    rc = tn_gemm(ctx, (const uint16_t*)B.H2, HID, (const uint16_t*)B.dY, K3, K3, rows_pad, 0, 0, part,
                 grads + OFF_W3, grads + OFF_B3, st);
    if (rc) return rc;
    if (loss) {
        k_mlp_loss<<<1, 256, 0, st>>>(B.loss, blocks, (float)(1.0 / (3.0 * (double)rows)), loss);
        SSS_LAUNCH_CHECK(ctx, "k_mlp_loss");
    }
    return SSS_OK;
}

extern "C" int sss_mlp_adam(sss_ctx* ctx, float* params, const float* grads, float* m, float* v, int64_t n, int t,
                            double lr, double beta1, double beta2, double eps, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (n < 0 || t < 1) return sss_set_err(ctx, SSS_ERR_ARG, "bad Adam arguments");
    if (n == 0) return SSS_OK;
    if (!params || !grads || !m || !v) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    // bias corrections folded into the step size and epsilon:
    // p -= lr * (m / c1) / (sqrt(v / c2) + eps) = lr_t * m / (sqrt(v) + eps * sqrt(c2))
    const double c1 = 1.0 - pow(beta1, t), c2 = 1.0 - pow(beta2, t);
    const double lr_t = lr * sqrt(c2) / c1;
    const double eps_t = eps * sqrt(c2);
    k_mlp_adam<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(params, grads, m, v, n, (float)lr_t,
                                                                             (float)beta1, (float)beta2, (float)eps_t);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_adam");
    return SSS_OK;
}
