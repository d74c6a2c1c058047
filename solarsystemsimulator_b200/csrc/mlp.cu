// Learned short-range correction of the 3-D mesh force: a per-particle MLP
// 67 -> 128 -> 128 -> 3 (SiLU), bf16 weights and activations on the tensor
// cores (mma.sync.m16n8k16 bf16 -> f32), trained online on the GPU by the
// kernels of this file.
//
// A warp owns 16 particles (rows). Layer outputs stay in registers: the f32
// accumulator fragments of two adjacent 8-column tiles are exactly the bf16
// A fragment of the next layer's 16-wide k tile, so a row never leaves the
// register file between its inputs and its outputs. Weights are pre-packed
// (sss_mlp_pack) into per-lane B fragments, staged once per CTA in shared
// memory and read as one 8-byte load per lane and mma.
//
// Training: k_mlp_rows runs forward and backward per 16-row tile (deltas
// through W3^T and W2^T in the same fragment scheme) and writes the
// activations and deltas the weight gradients need; k_mlp_tn forms
// dW = A^T dZ over the rows (transposed staging in shared memory, one
// m16 tile per warp, partial sums per CTA), and k_mlp_reduce adds the CTA
// partials in a fixed order, so gradients are deterministic. Rounding
// points: inputs, weights, hidden activations, output delta and hidden
// deltas are bf16; every sum is f32.

#include "pm3d.cuh"

#include <cuda_bf16.h>

#include <algorithm>

namespace {

constexpr int K1 = 80, HID = 128, K3 = 8;   // 67 inputs padded to 80
constexpr int KT1 = K1 / 16, KT2 = HID / 16, NTH = HID / 8;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + K1 * HID, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID;
constexpr int OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * K3, NPAR = OFF_B3 + K3;
constexpr int FR_W1 = 0, FR_W2 = FR_W1 + KT1 * NTH * 64, FR_W3 = FR_W2 + KT2 * NTH * 64;
constexpr int FR_W3T = FR_W3 + KT2 * 64, FR_W2T = FR_W3T + NTH * 64, NFR = FR_W2T + KT2 * NTH * 64;
static_assert(NPAR == SSS_MLP_N_PARAMS, "parameter layout");
static_assert(NFR == SSS_MLP_N_FRAGS, "fragment layout");
static_assert(K1 == SSS_MLP_IN_PAD, "input width");

constexpr int XS = 44;          // row stride (uint32) of a staged 16 x 80 bf16 input tile (88 bf16)
constexpr int WARPS_FWD = 8;    // warps per CTA of the forward kernels (sharing one weight copy)

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x (low half) = lo
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SiLU and its derivative with the fast exponential and division (both a few
// ulp; the result is rounded to bf16 or multiplied into a bf16 delta)
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------- packing

// One thread per uint32 of the fragment arrays. A B fragment of an operand
// B[k][n] for tile (kt, nt) and lane (g = lane / 4, t = lane % 4) is
// {B[16kt+2t][8nt+g], B[16kt+2t+1][8nt+g]} (register 0) and the same at
// rows +8 (register 1), lower k in the low half.
__global__ void k_mlp_pack(const float* __restrict__ P, uint32_t* __restrict__ F) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= NFR) return;
    int base, ntn;
    if (f < FR_W2) base = FR_W1, ntn = NTH;
    else if (f < FR_W3) base = FR_W2, ntn = NTH;
    else if (f < FR_W3T) base = FR_W3, ntn = 1;
    else if (f < FR_W2T) base = FR_W3T, ntn = NTH;
    else base = FR_W2T, ntn = NTH;
    const int l = f - base;
    const int r = l & 1, lane = (l >> 1) & 31, tile = l >> 6;
    const int kt = tile / ntn, nt = tile % ntn;
    const int g = lane >> 2, t = lane & 3;
    const int k0 = 16 * kt + 2 * t + 8 * r, n = 8 * nt + g;
    float lo, hi;
    if (base == FR_W1) {
        lo = P[OFF_W1 + k0 * HID + n];
        hi = P[OFF_W1 + (k0 + 1) * HID + n];
    } else if (base == FR_W2) {
        lo = P[OFF_W2 + k0 * HID + n];
        hi = P[OFF_W2 + (k0 + 1) * HID + n];
    } else if (base == FR_W3) {
        lo = P[OFF_W3 + k0 * K3 + n];
        hi = P[OFF_W3 + (k0 + 1) * K3 + n];
    } else if (base == FR_W3T) {       // B(k, n) = W3[n][k], k < 8
        lo = k0 < K3 ? P[OFF_W3 + n * K3 + k0] : 0.0f;
        hi = k0 + 1 < K3 ? P[OFF_W3 + n * K3 + k0 + 1] : 0.0f;
    } else {                           // B(k, n) = W2[n][k]
        lo = P[OFF_W2 + n * HID + k0];
        hi = P[OFF_W2 + n * HID + k0 + 1];
    }
    F[f] = pack2(lo, hi);
}

// ------------------------------------------------------------- features

// Inputs of one particle, written by the two lanes that share a row: half 0
// the cells with x offset -1, 0 (columns 0..31), half 1 the cells with x
// offset +1, +2 (32..63), the offsets t - 1/2 (64..66) and zeros (67..87).
__device__ __forceinline__ void particle_features(const float* __restrict__ rho, int n, double inv_h,
                                                  float inv_mean, const Pm3Parts& s, long long p, int half,
                                                  uint16_t* __restrict__ row) {
    if (p < 0) {
        for (int c = half * 44; c < half * 44 + 44; ++c) row[c] = 0;
        return;
    }
    int i[3];
    double t[3];
    for (int c = 0; c < 3; ++c) pm3_cell(s.x[c][p], inv_h, n, i[c], t[c]);
    // wrapped cell offsets of the patch, then all 32 loads in flight at once
    long long ox[2];
    int oy[4], oz[4];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        int ix = i[0] + 2 * half + a - 1;
        ix += ix < 0 ? n : 0;
        ix -= ix >= n ? n : 0;
        ox[a] = (long long)ix * n * n;
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        int iy = i[1] + b - 1, iz = i[2] + b - 1;
        iy += iy < 0 ? n : 0;
        iy -= iy >= n ? n : 0;
        iz += iz < 0 ? n : 0;
        iz -= iz >= n ? n : 0;
        oy[b] = iy * n;
        oz[b] = iz;
    }
    float v[32];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int e = 0; e < 4; ++e) v[a * 16 + b * 4 + e] = __ldg(rho + ox[a] + oy[b] + oz[e]);
#pragma unroll
    for (int q = 0; q < 32; q += 2) {
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(log1pf(v[q] * inv_mean), log1pf(v[q + 1] * inv_mean));
        *reinterpret_cast<__nv_bfloat162*>(row + half * 32 + q) = h2;
    }
    if (half == 1) {
        for (int c = 0; c < 3; ++c) row[64 + c] = __bfloat16_as_ushort(__float2bfloat16_rn((float)(t[c] - 0.5)));
        for (int c = 67; c < 88; ++c) row[c] = 0;
    }
}

// --------------------------------------------------------- forward (warp)

// Forward of the 16 rows staged in Xs (row stride XS uint32) with the
// fragments in sF and biases in sB (b1 | b2 | b3); Ys[16][4] receives the
// outputs (columns 0..2 valid).
__device__ __forceinline__ void tile_forward(const uint32_t* __restrict__ sF, const float* __restrict__ sB,
                                             const uint32_t* __restrict__ Xs, float* __restrict__ Ys) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[NTH][4];
    uint32_t h[KT2][4];
#pragma unroll
    for (int nt = 0; nt < NTH; ++nt) {
        const float b0 = sB[8 * nt + 2 * t], b1 = sB[8 * nt + 2 * t + 1];
        acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < KT1; ++kt) {
        uint32_t a[4];
        a[0] = Xs[g * XS + kt * 8 + t];
        a[1] = Xs[(g + 8) * XS + kt * 8 + t];
        a[2] = Xs[g * XS + kt * 8 + 4 + t];
        a[3] = Xs[(g + 8) * XS + kt * 8 + 4 + t];
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W1 + ((kt * NTH + nt) * 32 + lane) * 2);
            mma16816(acc[nt], a, b.x, b.y);
        }
    }
#pragma unroll
    for (int k = 0; k < KT2; ++k) {
        h[k][0] = pack2(silu(acc[2 * k][0]), silu(acc[2 * k][1]));
        h[k][1] = pack2(silu(acc[2 * k][2]), silu(acc[2 * k][3]));
        h[k][2] = pack2(silu(acc[2 * k + 1][0]), silu(acc[2 * k + 1][1]));
        h[k][3] = pack2(silu(acc[2 * k + 1][2]), silu(acc[2 * k + 1][3]));
    }
#pragma unroll
    for (int nt = 0; nt < NTH; ++nt) {
        const float b0 = sB[HID + 8 * nt + 2 * t], b1 = sB[HID + 8 * nt + 2 * t + 1];
        acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < KT2; ++kt)
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W2 + ((kt * NTH + nt) * 32 + lane) * 2);
            mma16816(acc[nt], h[kt], b.x, b.y);
        }
#pragma unroll
    for (int k = 0; k < KT2; ++k) {
        h[k][0] = pack2(silu(acc[2 * k][0]), silu(acc[2 * k][1]));
        h[k][1] = pack2(silu(acc[2 * k][2]), silu(acc[2 * k][3]));
        h[k][2] = pack2(silu(acc[2 * k + 1][0]), silu(acc[2 * k + 1][1]));
        h[k][3] = pack2(silu(acc[2 * k + 1][2]), silu(acc[2 * k + 1][3]));
    }
    float o[4];
    o[0] = sB[2 * HID + 2 * t]; o[1] = sB[2 * HID + 2 * t + 1]; o[2] = o[0]; o[3] = o[1];
#pragma unroll
    for (int kt = 0; kt < KT2; ++kt) {
        const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W3 + (kt * 32 + lane) * 2);
        mma16816(o, h[kt], b.x, b.y);
    }
    if (t < 2) {
        Ys[g * 4 + 2 * t] = o[0];
        Ys[g * 4 + 2 * t + 1] = o[1];
        Ys[(g + 8) * 4 + 2 * t] = o[2];
        Ys[(g + 8) * 4 + 2 * t + 1] = o[3];
    }
}

// shared memory of the forward kernels: fragments W1 W2 W3, biases, per
// warp an input tile and an output tile
constexpr int FWD_SMEM_U32 = FR_W3T + 2 * HID + K3 + WARPS_FWD * (16 * XS + 16 * 4);

__device__ __forceinline__ void stage_forward_weights(const float* __restrict__ P, const uint32_t* __restrict__ F,
                                                      uint32_t* sF, float* sB) {
    for (int i = threadIdx.x; i < FR_W3T / 4; i += blockDim.x)
        reinterpret_cast<uint4*>(sF)[i] = reinterpret_cast<const uint4*>(F)[i];
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        sB[i] = P[OFF_B1 + i];
        sB[HID + i] = P[OFF_B2 + i];
    }
    if (threadIdx.x < K3) sB[2 * HID + threadIdx.x] = P[OFF_B3 + threadIdx.x];
}

// ------------------------------------------- correction pass on tcgen05

// The correction pass with layers 1 and 2 on the 5th-generation tensor
// cores: one CTA of 128 threads owns a tile of 128 particles (one particle
// per thread = one TMEM lane). Operands live in shared memory in the
// canonical no-swizzle K-major layout (8-row x 16-byte core matrices,
// K-adjacent core matrices 128 bytes apart, 8-row groups K*16 bytes apart);
// one thread issues tcgen05.mma (M = N = 128, K = 16 per instruction) into
// f32 accumulators in TMEM (256 columns: layer 1 | layer 2), tcgen05.commit
// signals an mbarrier, and every thread reads its own row back with
// tcgen05.ld for bias + SiLU (bf16 row of the next operand) or, after layer
// 2, for the 128 x 3 output layer on the CUDA cores and the KDK epilogue.
// The rounding points are those of the mma.sync kernels (bf16 inputs,
// weights and hidden activations; f32 sums). Waits are bounded; the TMEM
// columns are freed on every path.
namespace tc {
constexpr int ROWS = 128;
constexpr int OFF_W1 = 0;                          // W1^T: 128 x 80 bf16 (B operand, rows = outputs)
constexpr int OFF_W2 = OFF_W1 + HID * K1 * 2;      // W2^T: 128 x 128 bf16
constexpr int OFF_X = OFF_W2 + HID * HID * 2;      // inputs: 128 x 80 bf16 (A operand, rows = particles)
constexpr int OFF_H = OFF_X + ROWS * K1 * 2;       // hidden 1: 128 x 128 bf16
constexpr int OFF_F = OFF_H + ROWS * HID * 2;      // f32: b1[128] b2[128] b3[8] W3[128][3]
constexpr int N_F = HID + HID + K3 + HID * 3;
constexpr int OFF_BAR = (OFF_F + N_F * 4 + 15) / 16 * 16;
constexpr int SMEM = OFF_BAR + 16;
constexpr uint32_t TMEM_COLS = 256;
// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, N = 128, M = 128
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 >> 3) << 17) |
                           ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ int canon(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor: start, leading offset (K direction) 128 B,
// stride offset (8-row groups) K * 16 B, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t desc(uint32_t saddr, int K) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)((K * 16) >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[M x K] B[N x K]^T over K / 16 instructions, then commit to bar
__device__ __forceinline__ void mma_layer(uint32_t tmem_d, uint32_t sa, uint32_t sb, int K, uint64_t* bar) {
    for (int kk = 0; kk < K / 16; ++kk) {
        const uint64_t da = desc(sa + kk * 256, K), db = desc(sb + kk * 256, K);
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            :: "r"(tmem_d), "l"(da), "l"(db), "r"(IDESC), "r"(kk) : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(sss_smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld32_nowait(uint32_t addr, float (&v)[32]) {
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
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
}  // namespace tc

// inputs of particle p (p >= n: zeros) into row r of the canonical X tile
__device__ __forceinline__ void tc_features(const Pm3Parts& s, const float* __restrict__ rho, int n, double inv_h,
                                            float inv_mean, long long p, int r, uint8_t* sx) {
    uint32_t row[K1 / 2];
#pragma unroll
    for (int q = 0; q < K1 / 2; ++q) row[q] = 0u;
    if (p < s.n) {
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
        float v[64];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int c = 0; c < 4; ++c) v[a * 16 + b * 4 + c] = __ldg(rho + ox[a] + oy[b] + oz[c]);
#pragma unroll
        for (int q = 0; q < 32; ++q) row[q] = pack2(log1pf(v[2 * q] * inv_mean), log1pf(v[2 * q + 1] * inv_mean));
        row[32] = pack2((float)(t[0] - 0.5), (float)(t[1] - 0.5));
        row[33] = pack2((float)(t[2] - 0.5), 0.0f);
    }
#pragma unroll
    for (int j = 0; j < K1 / 8; ++j)
        *reinterpret_cast<uint4*>(sx + tc::canon(r, 8 * j, K1)) =
            make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
}

__global__ void __launch_bounds__(tc::ROWS, 2) k_mlp_correct_tc(const Pm3Parts s, const float* __restrict__ rho,
                                                                int n, double inv_h, float inv_mean,
                                                                const float* __restrict__ P, double out_scale,
                                                                const Pm3Epi e, int* status) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    float* sFl = reinterpret_cast<float*>(sm + tc::OFF_F);
    float* sb1 = sFl;
    float* sb2 = sFl + HID;
    float* sb3 = sFl + 2 * HID;
    float* sW3 = sFl + 2 * HID + K3;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + tc::OFF_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + tc::OFF_BAR + 8);
    // weights in the canonical layout (W^T: row = output unit, K = input)
    for (int i = tid; i < K1 * HID; i += blockDim.x) {
        const int k = i / HID, c = i % HID;
        *reinterpret_cast<__nv_bfloat16*>(sm + tc::OFF_W1 + tc::canon(c, k, K1)) =
            __float2bfloat16_rn(P[OFF_W1 + i]);
    }
    for (int i = tid; i < HID * HID; i += blockDim.x) {
        const int k = i / HID, c = i % HID;
        *reinterpret_cast<__nv_bfloat16*>(sm + tc::OFF_W2 + tc::canon(c, k, HID)) =
            __float2bfloat16_rn(P[OFF_W2 + i]);
    }
    for (int i = tid; i < HID; i += blockDim.x) {
        sb1[i] = P[OFF_B1 + i];
        sb2[i] = P[OFF_B2 + i];
        for (int c = 0; c < 3; ++c) sW3[i * 3 + c] = __bfloat162float(__float2bfloat16_rn(P[OFF_W3 + i * K3 + c]));
    }
    if (tid < K3) sb3[tid] = P[OFF_B3 + tid];
    if (tid == 0) {
        sss_mbar_init(bar, 1);
        sss_fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(sss_smem_addr(tslot)), "r"(tc::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_smem_to_async();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t d1 = tmem, d2 = tmem + HID;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    const uint32_t sX = sss_smem_addr(sm + tc::OFF_X), sH = sss_smem_addr(sm + tc::OFF_H);
    const uint32_t sW1 = sss_smem_addr(sm + tc::OFF_W1), sW2 = sss_smem_addr(sm + tc::OFF_W2);
    unsigned phase = 0;
    const long long tiles = (s.n + tc::ROWS - 1) / tc::ROWS;
    if (blockIdx.x < tiles) tc_features(s, rho, n, inv_h, inv_mean, (long long)blockIdx.x * tc::ROWS + tid, tid,
                                        sm + tc::OFF_X);
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long p = tile * tc::ROWS + tid;
        tc::fence_smem_to_async();
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        // ---- layer 1 on the tensor cores
        if (tid == 0) tc::mma_layer(d1, sX, sW1, K1, bar);
        int bad = sss_mbar_wait_bounded(bar, phase, status) ? 0 : 1;
        phase ^= 1u;
        if (__syncthreads_or(bad)) break;
        tc::fence_after();
#pragma unroll 1
        for (int j2 = 0; j2 < HID / 64; ++j2) {
            float v[2][32];
            tc::tmem_ld32_nowait(d1 + lane_base + 64 * j2, v[0]);
            tc::tmem_ld32_nowait(d1 + lane_base + 64 * j2 + 32, v[1]);
            tc::tmem_wait_ld();
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int j = 2 * j2 + hh;
                uint32_t h[16];
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    h[q] = pack2(silu(v[hh][2 * q] + sb1[32 * j + 2 * q]),
                                 silu(v[hh][2 * q + 1] + sb1[32 * j + 2 * q + 1]));
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    *reinterpret_cast<uint4*>(sm + tc::OFF_H + tc::canon(tid, 32 * j + 8 * u, HID)) =
                        make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
            }
        }
        tc::fence_smem_to_async();
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        // ---- layer 2 on the tensor cores
        if (tid == 0) tc::mma_layer(d2, sH, sW2, HID, bar);
        // the input tile is free once layer 1 has completed: gather the next
        // tile's inputs while layer 2 runs
        if (tile + gridDim.x < tiles)
            tc_features(s, rho, n, inv_h, inv_mean, (tile + gridDim.x) * tc::ROWS + tid, tid, sm + tc::OFF_X);
        bad = sss_mbar_wait_bounded(bar, phase, status) ? 0 : 1;
        phase ^= 1u;
        if (__syncthreads_or(bad)) break;
        tc::fence_after();
        float y0 = sb3[0], y1 = sb3[1], y2 = sb3[2];
#pragma unroll 1
        for (int j2 = 0; j2 < HID / 64; ++j2) {
            float v[2][32];
            tc::tmem_ld32_nowait(d2 + lane_base + 64 * j2, v[0]);
            tc::tmem_ld32_nowait(d2 + lane_base + 64 * j2 + 32, v[1]);
            tc::tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 64; ++q) {
                const int k = 64 * j2 + q;
                const float hq = __bfloat162float(__float2bfloat16_rn(silu(v[q >> 5][q & 31] + sb2[k])));
                y0 = fmaf(hq, sW3[3 * k], y0);
                y1 = fmaf(hq, sW3[3 * k + 1], y1);
                y2 = fmaf(hq, sW3[3 * k + 2], y2);
            }
        }
        if (p < s.n) {
            const double ax = s.a[0][p] + out_scale * (double)y0;
            const double ay = s.a[1][p] + out_scale * (double)y1;
            const double az = s.a[2][p] + out_scale * (double)y2;
            pm3_epilogue(s, e, p, ax, ay, az);
        }
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(tc::TMEM_COLS)
                     : "memory");
}

// forward on given input rows (sss_mlp_forward)
__global__ void __launch_bounds__(WARPS_FWD * 32, 2) k_mlp_fwd(const uint16_t* __restrict__ X, long long rows,
                                                            const float* __restrict__ P,
                                                            const uint32_t* __restrict__ F, float* __restrict__ Y) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* sF = smem;
    float* sB = reinterpret_cast<float*>(smem + FR_W3T);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* Xs = smem + FR_W3T + 2 * HID + K3 + warp * (16 * XS + 16 * 4);
    float* Ys = reinterpret_cast<float*>(Xs + 16 * XS);
    stage_forward_weights(P, F, sF, sB);
    __syncthreads();
    const uint32_t* X32 = reinterpret_cast<const uint32_t*>(X);
    const long long tiles = (rows + 15) / 16;
    for (long long tile = (long long)blockIdx.x * WARPS_FWD + warp; tile < tiles;
         tile += (long long)gridDim.x * WARPS_FWD) {
        for (int i = lane; i < 16 * (K1 / 2); i += 32) {
            const int r = i / (K1 / 2), c = i % (K1 / 2);
            const long long row = tile * 16 + r;
            Xs[r * XS + c] = row < rows ? X32[row * (K1 / 2) + c] : 0u;
        }
        __syncwarp();
        tile_forward(sF, sB, Xs, Ys);
        __syncwarp();
        if (lane < 16) {
            const long long row = tile * 16 + lane;
            if (row < rows)
                for (int c = 0; c < 3; ++c) Y[row * 3 + c] = Ys[lane * 4 + c];
        }
        __syncwarp();
    }
}

// features of selected particles (sss_mlp_features)
__global__ void k_mlp_features(const Pm3Parts s, const float* __restrict__ rho, int n, double inv_h, float inv_mean,
                               const long long* __restrict__ idx, long long rows, uint16_t* __restrict__ X) {
    __shared__ __align__(16) uint16_t tile[4][16][88];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long r = ((long long)blockIdx.x * 4 + warp) * 16 + (lane & 15);
    long long p = -1;
    if (r < rows) p = idx ? idx[r] : r;
    if (p >= s.n) p = -1;
    particle_features(rho, n, inv_h, inv_mean, s, p, lane >> 4, tile[warp][lane & 15]);
    __syncwarp();
    if (r < rows)
        for (int c = (lane >> 4) * 40; c < (lane >> 4) * 40 + 40; ++c) X[r * K1 + c] = tile[warp][lane & 15][c];
}

// ------------------------------------------------------------- training

struct RowBufs {
    uint32_t* Xc;       // [rows_pad][40] compacted inputs (when idx is given)
    uint32_t* H1;       // [rows_pad][64] bf16 pairs
    uint32_t* H2;
    uint32_t* dZ1;
    uint32_t* dZ2;
    uint32_t* dY;       // [rows_pad][4]
    float* G1;          // [rows_pad][128] silu'(Z1)
    float* G2;
    float* loss;        // [tiles]
};

constexpr int ROWS_WARPS = 4;
constexpr int ROWS_SMEM_U32 = NFR + 2 * HID + K3;

__global__ void __launch_bounds__(ROWS_WARPS * 32) k_mlp_rows(const uint16_t* __restrict__ X,
                                                              const float* __restrict__ T,
                                                              const int* __restrict__ idx, long long rows,
                                                              long long x_rows, long long rows_pad, float dscale,
                                                              const float* __restrict__ P,
                                                              const uint32_t* __restrict__ F, const RowBufs B) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* sF = smem;
    float* sB = reinterpret_cast<float*>(smem + NFR);
    for (int i = threadIdx.x; i < NFR / 4; i += blockDim.x)
        reinterpret_cast<uint4*>(sF)[i] = reinterpret_cast<const uint4*>(F)[i];
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        sB[i] = P[OFF_B1 + i];
        sB[HID + i] = P[OFF_B2 + i];
    }
    if (threadIdx.x < K3) sB[2 * HID + threadIdx.x] = P[OFF_B3 + threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const uint32_t* X32 = reinterpret_cast<const uint32_t*>(X);
    const long long tiles = rows_pad / 16;
    for (long long tile = (long long)blockIdx.x * ROWS_WARPS + warp; tile < tiles;
         tile += (long long)gridDim.x * ROWS_WARPS) {
        const long long r0 = tile * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < rows, v1 = r1 < rows;
        long long s0 = v0 ? (idx ? (long long)idx[r0] : r0) : -1;
        long long s1 = v1 ? (idx ? (long long)idx[r1] : r1) : -1;
        if (s0 >= x_rows) s0 = -1;      // an index outside X reads as a zero row with no target
        if (s1 >= x_rows) s1 = -1;
        float acc[NTH][4];
        uint32_t h[KT2][4];
        // ---- layer 1
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const float b0 = sB[8 * nt + 2 * t], b1 = sB[8 * nt + 2 * t + 1];
            acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
        }
#pragma unroll
        for (int kt = 0; kt < KT1; ++kt) {
            uint32_t a[4];
            a[0] = s0 >= 0 ? X32[s0 * 40 + kt * 8 + t] : 0u;
            a[1] = s1 >= 0 ? X32[s1 * 40 + kt * 8 + t] : 0u;
            a[2] = s0 >= 0 ? X32[s0 * 40 + kt * 8 + 4 + t] : 0u;
            a[3] = s1 >= 0 ? X32[s1 * 40 + kt * 8 + 4 + t] : 0u;
            if (B.Xc) {
                B.Xc[r0 * 40 + kt * 8 + t] = a[0];
                B.Xc[r1 * 40 + kt * 8 + t] = a[1];
                B.Xc[r0 * 40 + kt * 8 + 4 + t] = a[2];
                B.Xc[r1 * 40 + kt * 8 + 4 + t] = a[3];
            }
#pragma unroll
            for (int nt = 0; nt < NTH; ++nt) {
                const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W1 + ((kt * NTH + nt) * 32 + lane) * 2);
                mma16816(acc[nt], a, b.x, b.y);
            }
        }
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const int c = 8 * nt + 2 * t;
            *reinterpret_cast<float2*>(B.G1 + r0 * HID + c) = make_float2(dsilu(acc[nt][0]), dsilu(acc[nt][1]));
            *reinterpret_cast<float2*>(B.G1 + r1 * HID + c) = make_float2(dsilu(acc[nt][2]), dsilu(acc[nt][3]));
        }
#pragma unroll
        for (int k = 0; k < KT2; ++k) {
            h[k][0] = pack2(silu(acc[2 * k][0]), silu(acc[2 * k][1]));
            h[k][1] = pack2(silu(acc[2 * k][2]), silu(acc[2 * k][3]));
            h[k][2] = pack2(silu(acc[2 * k + 1][0]), silu(acc[2 * k + 1][1]));
            h[k][3] = pack2(silu(acc[2 * k + 1][2]), silu(acc[2 * k + 1][3]));
            B.H1[r0 * 64 + k * 8 + t] = h[k][0];
            B.H1[r1 * 64 + k * 8 + t] = h[k][1];
            B.H1[r0 * 64 + k * 8 + 4 + t] = h[k][2];
            B.H1[r1 * 64 + k * 8 + 4 + t] = h[k][3];
        }
        // ---- layer 2
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const float b0 = sB[HID + 8 * nt + 2 * t], b1 = sB[HID + 8 * nt + 2 * t + 1];
            acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
        }
#pragma unroll
        for (int kt = 0; kt < KT2; ++kt)
#pragma unroll
            for (int nt = 0; nt < NTH; ++nt) {
                const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W2 + ((kt * NTH + nt) * 32 + lane) * 2);
                mma16816(acc[nt], h[kt], b.x, b.y);
            }
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const int c = 8 * nt + 2 * t;
            *reinterpret_cast<float2*>(B.G2 + r0 * HID + c) = make_float2(dsilu(acc[nt][0]), dsilu(acc[nt][1]));
            *reinterpret_cast<float2*>(B.G2 + r1 * HID + c) = make_float2(dsilu(acc[nt][2]), dsilu(acc[nt][3]));
        }
#pragma unroll
        for (int k = 0; k < KT2; ++k) {
            h[k][0] = pack2(silu(acc[2 * k][0]), silu(acc[2 * k][1]));
            h[k][1] = pack2(silu(acc[2 * k][2]), silu(acc[2 * k][3]));
            h[k][2] = pack2(silu(acc[2 * k + 1][0]), silu(acc[2 * k + 1][1]));
            h[k][3] = pack2(silu(acc[2 * k + 1][2]), silu(acc[2 * k + 1][3]));
            B.H2[r0 * 64 + k * 8 + t] = h[k][0];
            B.H2[r1 * 64 + k * 8 + t] = h[k][1];
            B.H2[r0 * 64 + k * 8 + 4 + t] = h[k][2];
            B.H2[r1 * 64 + k * 8 + 4 + t] = h[k][3];
        }
        // ---- layer 3 and the output delta
        float o[4];
        o[0] = sB[2 * HID + 2 * t]; o[1] = sB[2 * HID + 2 * t + 1]; o[2] = o[0]; o[3] = o[1];
#pragma unroll
        for (int kt = 0; kt < KT2; ++kt) {
            const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W3 + (kt * 32 + lane) * 2);
            mma16816(o, h[kt], b.x, b.y);
        }
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        float l2 = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int col = 2 * t + (q & 1);
            const long long sr = (q < 2) ? s0 : s1;      // source row of X and T
            if (sr >= 0 && col < 3) {
                const float e = o[q] - T[sr * 3 + col];
                d[q] = dscale * e;
                l2 += e * e;
            }
        }
        uint32_t ad[4];
        ad[0] = pack2(d[0], d[1]);
        ad[1] = pack2(d[2], d[3]);
        ad[2] = 0u;
        ad[3] = 0u;
        B.dY[r0 * 4 + t] = ad[0];
        B.dY[r1 * 4 + t] = ad[1];
        // ---- dZ2 = (dY W3^T) * silu'(Z2)
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
            const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W3T + (nt * 32 + lane) * 2);
            mma16816(acc[nt], ad, b.x, b.y);
        }
#pragma unroll
        for (int k = 0; k < KT2; ++k) {
            float gz[2][4];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int c = 8 * (2 * k + u) + 2 * t;
                const float2 q0 = *reinterpret_cast<const float2*>(B.G2 + r0 * HID + c);
                const float2 q1 = *reinterpret_cast<const float2*>(B.G2 + r1 * HID + c);
                gz[u][0] = acc[2 * k + u][0] * q0.x;
                gz[u][1] = acc[2 * k + u][1] * q0.y;
                gz[u][2] = acc[2 * k + u][2] * q1.x;
                gz[u][3] = acc[2 * k + u][3] * q1.y;
            }
            h[k][0] = pack2(gz[0][0], gz[0][1]);
            h[k][1] = pack2(gz[0][2], gz[0][3]);
            h[k][2] = pack2(gz[1][0], gz[1][1]);
            h[k][3] = pack2(gz[1][2], gz[1][3]);
            B.dZ2[r0 * 64 + k * 8 + t] = h[k][0];
            B.dZ2[r1 * 64 + k * 8 + t] = h[k][1];
            B.dZ2[r0 * 64 + k * 8 + 4 + t] = h[k][2];
            B.dZ2[r1 * 64 + k * 8 + 4 + t] = h[k][3];
        }
        // ---- dZ1 = (dZ2 W2^T) * silu'(Z1)
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < KT2; ++kt)
#pragma unroll
            for (int nt = 0; nt < NTH; ++nt) {
                const uint2 b = *reinterpret_cast<const uint2*>(sF + FR_W2T + ((kt * NTH + nt) * 32 + lane) * 2);
                mma16816(acc[nt], h[kt], b.x, b.y);
            }
#pragma unroll
        for (int nt = 0; nt < NTH; ++nt) {
            const int c = 8 * nt + 2 * t;
            const float2 q0 = *reinterpret_cast<const float2*>(B.G1 + r0 * HID + c);
            const float2 q1 = *reinterpret_cast<const float2*>(B.G1 + r1 * HID + c);
            B.dZ1[r0 * 64 + c / 2] = pack2(acc[nt][0] * q0.x, acc[nt][1] * q0.y);
            B.dZ1[r1 * 64 + c / 2] = pack2(acc[nt][2] * q1.x, acc[nt][3] * q1.y);
        }
        // ---- loss partial of the tile
#pragma unroll
        for (int off = 16; off; off >>= 1) l2 += __shfl_xor_sync(0xffffffffu, l2, off);
        if (lane == 0) B.loss[tile] = l2;
    }
}

// dW = A^T Bm over S rows: A [S][lda] bf16 (M columns used), Bm [S][ldb]
// bf16 (N = 8 * NTN columns); each CTA sums its rows [c * per, (c+1) * per)
// into part[c][M * N] and the column sums of Bm into part[c][M * N + n].
constexpr int TN_ROWS = 64;                  // rows staged per round
constexpr int TN_LD = TN_ROWS + 8;           // bf16 row stride of the transposed tiles

template <int NTN>
__global__ void __launch_bounds__(256) k_mlp_tn(const uint16_t* __restrict__ A, int lda, int M,
                                                const uint16_t* __restrict__ Bm, int ldb, long long S,
                                                long long per, float* __restrict__ part) {
    constexpr int N = 8 * NTN;
    __shared__ __align__(16) uint16_t sA[HID][TN_LD];
    __shared__ __align__(16) uint16_t sBt[N][TN_LD];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long r0 = (long long)blockIdx.x * per;
    const long long r1 = min(S, r0 + per);
    float acc[NTN][4];
#pragma unroll
    for (int nt = 0; nt < NTN; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
    float cs = 0.0f;
    const bool active = warp * 16 < M;
    for (long long b = r0; b < r1; b += TN_ROWS) {
        __syncthreads();
        for (int i = threadIdx.x; i < TN_ROWS * (M / 2); i += blockDim.x) {
            const int rl = i / (M / 2), mp = i % (M / 2);
            const long long row = b + rl;
            uint32_t v = 0u;
            if (row < r1) v = *reinterpret_cast<const uint32_t*>(A + row * lda + 2 * mp);
            sA[2 * mp][rl] = (uint16_t)(v & 0xffffu);
            sA[2 * mp + 1][rl] = (uint16_t)(v >> 16);
        }
        for (int i = threadIdx.x; i < TN_ROWS * (N / 2); i += blockDim.x) {
            const int rl = i / (N / 2), np = i % (N / 2);
            const long long row = b + rl;
            uint32_t v = 0u;
            if (row < r1) v = *reinterpret_cast<const uint32_t*>(Bm + row * ldb + 2 * np);
            sBt[2 * np][rl] = (uint16_t)(v & 0xffffu);
            sBt[2 * np + 1][rl] = (uint16_t)(v >> 16);
        }
        __syncthreads();
        if (threadIdx.x < N)
            for (int rl = 0; rl < TN_ROWS; ++rl) cs += __bfloat162float(__ushort_as_bfloat16(sBt[threadIdx.x][rl]));
        if (active) {
            const uint32_t* a32 = reinterpret_cast<const uint32_t*>(&sA[0][0]);
            const uint32_t* b32 = reinterpret_cast<const uint32_t*>(&sBt[0][0]);
            constexpr int LD32 = TN_LD / 2;
#pragma unroll
            for (int kk = 0; kk < TN_ROWS / 16; ++kk) {
                uint32_t a[4];
                a[0] = a32[(16 * warp + g) * LD32 + kk * 8 + t];
                a[1] = a32[(16 * warp + g + 8) * LD32 + kk * 8 + t];
                a[2] = a32[(16 * warp + g) * LD32 + kk * 8 + 4 + t];
                a[3] = a32[(16 * warp + g + 8) * LD32 + kk * 8 + 4 + t];
#pragma unroll
                for (int nt = 0; nt < NTN; ++nt) {
                    const uint32_t b0 = b32[(8 * nt + g) * LD32 + kk * 8 + t];
                    const uint32_t b1 = b32[(8 * nt + g) * LD32 + kk * 8 + 4 + t];
                    mma16816(acc[nt], a, b0, b1);
                }
            }
        }
    }
    float* out = part + (long long)blockIdx.x * (M * N + N);
    if (active) {
#pragma unroll
        for (int nt = 0; nt < NTN; ++nt) {
            const int c = 8 * nt + 2 * t;
            out[(16 * warp + g) * N + c] = acc[nt][0];
            out[(16 * warp + g) * N + c + 1] = acc[nt][1];
            out[(16 * warp + g + 8) * N + c] = acc[nt][2];
            out[(16 * warp + g + 8) * N + c + 1] = acc[nt][3];
        }
    }
    if (threadIdx.x < N) out[M * N + threadIdx.x] = cs;
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

__global__ void k_mlp_loss(const float* __restrict__ part, long long tiles, float scale, float* __restrict__ loss) {
    float s = 0.0f;
    for (long long i = threadIdx.x; i < tiles; i += blockDim.x) s += part[i];
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

int tn_gemm(sss_ctx* ctx, const uint16_t* A, int lda, int M, const uint16_t* Bm, int ldb, int N, long long S,
            float* part, float* gW, float* gb, int max_ctas, cudaStream_t st) {
    const long long per0 = (S + max_ctas - 1) / max_ctas;
    const long long per = std::max<long long>(TN_ROWS, (per0 + TN_ROWS - 1) / TN_ROWS * TN_ROWS);
    const int ctas = (int)std::max<long long>(1, (S + per - 1) / per);
    if (N == HID) k_mlp_tn<NTH><<<ctas, 256, 0, st>>>(A, lda, M, Bm, ldb, S, per, part);
    else k_mlp_tn<1><<<ctas, 256, 0, st>>>(A, lda, M, Bm, ldb, S, per, part);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_tn");
    const int tot = M * N + N;
    k_mlp_reduce<<<(tot + 255) / 256, 256, 0, st>>>(part, ctas, M * N, N, gW, gb);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_reduce");
    return SSS_OK;
}

}  // namespace

extern "C" int sss_mlp_pack(sss_ctx* ctx, const float* params, uint32_t* frags, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!params || !frags) return sss_set_err(ctx, SSS_ERR_ARG, "NULL parameters or fragments");
    k_mlp_pack<<<(NFR + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, frags);
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
    const unsigned blocks = (unsigned)((rows + 63) / 64);
    k_mlp_features<<<blocks, 128, 0, (cudaStream_t)stream>>>(pm3_parts(s), p->rho, p->n, p->n / p->box,
                                                            (float)(1.0 / rho_mean), (const long long*)idx, rows, X);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_features");
    return SSS_OK;
}

extern "C" int sss_mlp_forward(sss_ctx* ctx, const float* params, const uint32_t* frags, const uint16_t* X,
                               int64_t rows, float* Y, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (rows < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative row count");
    if (rows == 0) return SSS_OK;
    if (!params || !frags || !X || !Y) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    const size_t smem = FWD_SMEM_U32 * sizeof(uint32_t);
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long tiles = (rows + 15) / 16;
    const int blocks = (int)std::min<long long>((tiles + WARPS_FWD - 1) / WARPS_FWD, (long long)ctx->num_sms * 2);
    k_mlp_fwd<<<blocks, WARPS_FWD * 32, smem, (cudaStream_t)stream>>>(X, rows, params, frags, Y);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_fwd");
    return SSS_OK;
}

extern "C" int sss_mlp_correct(sss_ctx* ctx, sss_pm3* p, const sss_pm3_particles* s, const float* params,
                               const uint32_t* frags, double rho_mean, double out_scale, int mode, double hdt,
                               double dt, float* snap, void* stream) {
    if (!ctx || !p || !s) return SSS_ERR_ARG;
    if (s->n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative particle count");
    if (s->n == 0) return SSS_OK;
    if (!params || !frags) return sss_set_err(ctx, SSS_ERR_ARG, "NULL parameters or fragments");
    for (int c = 0; c < 3; ++c)
        if (!s->x[c] || !s->v[c] || !s->a[c]) return sss_set_err(ctx, SSS_ERR_ARG, "NULL particle array");
    if (!(rho_mean > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "rho_mean must be > 0");
    if (mode < SSS_PM3_FORCE || mode > SSS_PM3_KICK_DRIFT) return sss_set_err(ctx, SSS_ERR_ARG, "bad mode");
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_correct_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM));
    const long long tiles = (s->n + tc::ROWS - 1) / tc::ROWS;
    const int blocks = (int)std::min<long long>(tiles, (long long)ctx->num_sms * 2);
    Pm3Epi e{mode, hdt, dt, p->box, snap};
    k_mlp_correct_tc<<<blocks, tc::ROWS, tc::SMEM, (cudaStream_t)stream>>>(
        pm3_parts(s), p->rho, p->n, p->n / p->box, (float)(1.0 / rho_mean), params, out_scale, e, ctx->d_status);
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
    const long long rows_pad = (rows + 15) / 16 * 16;
    const long long tiles = rows_pad / 16;
    const int max_ctas = ctx->num_sms;
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
    const size_t oG1 = take((size_t)rows_pad * HID * 4), oG2 = take((size_t)rows_pad * HID * 4);
    const size_t oL = take((size_t)tiles * 4);
    const size_t oP = take((size_t)max_ctas * (HID * HID + HID) * 4);
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
    B.G1 = (float*)(base + oG1);
    B.G2 = (float*)(base + oG2);
    B.loss = (float*)(base + oL);
    float* part = (float*)(base + oP);
    const size_t smem = ROWS_SMEM_U32 * sizeof(uint32_t);
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (int)std::min<long long>((tiles + ROWS_WARPS - 1) / ROWS_WARPS, (long long)ctx->num_sms * 2);
    const float dscale = (float)(2.0 / (3.0 * (double)rows));
    k_mlp_rows<<<blocks, ROWS_WARPS * 32, smem, st>>>(X, T, idx, rows, x_rows, rows_pad, dscale, params, frags, B);
    SSS_LAUNCH_CHECK(ctx, "k_mlp_rows");
    const uint16_t* Xg = idx ? (const uint16_t*)B.Xc : X;
    // X rows beyond `rows` are read only when idx is NULL; pad rows of the
    // deltas are zero, so those products vanish, but the reads must stay in
    // the caller's array: use S = rows there
    const long long S1 = idx ? rows_pad : rows;
    rc = tn_gemm(ctx, Xg, K1, K1, (const uint16_t*)B.dZ1, HID, HID, S1, part, grads + OFF_W1, grads + OFF_B1,
                 max_ctas, st);
    if (rc) return rc;
    rc = tn_gemm(ctx, (const uint16_t*)B.H1, HID, HID, (const uint16_t*)B.dZ2, HID, HID, rows_pad, part,
                 grads + OFF_W2, grads + OFF_B2, max_ctas, st);
    if (rc) return rc;
    rc = tn_gemm(ctx, (const uint16_t*)B.H2, HID, HID, (const uint16_t*)B.dY, K3, K3, rows_pad, part,
                 grads + OFF_W3, grads + OFF_B3, max_ctas, st);
    if (rc) return rc;
    if (loss) {
        k_mlp_loss<<<1, 256, 0, st>>>(B.loss, tiles, (float)(1.0 / (3.0 * (double)rows)), loss);
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
