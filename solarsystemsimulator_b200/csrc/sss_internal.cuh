// Internal helpers shared by the libsss translation units: the context,
// error plumbing, and the sm_100a primitives (mbarrier, bulk async copy,
// bounded waits) the kernels are built from.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>
#include <string.h>

#include "../../include/sss.h"

struct sss_ctx {
    int device;
    int num_sms;
    char err[512];
    // scratch owned by the context (grown on demand, freed by sss_destroy)
    void* scratch;
    size_t scratch_bytes;
    // device status word written by bounded waits (SSS_ERR_TIMEOUT ...)
    int* d_status;
    // chunk-arrival counters of the all-pairs kernels (kept zero between
    // launches: the last chunk of a target block resets its counter)
    unsigned* d_counters;
    size_t n_counters;
    // cached CTAs-per-SM of the all-pairs kernels (0 = not yet queried)
    int occ[8];
    // the broadphase pipeline as an instantiated graph (broadphase.cu)
    struct sss_bp_graph* bp_graph;
};

void sss_bp_graph_free(struct sss_bp_graph* g);

int sss_set_err(sss_ctx* ctx, int code, const char* fmt, ...);
int sss_cuda_err(sss_ctx* ctx, cudaError_t e, const char* what);
// Ensure ctx->scratch holds at least `bytes` (256-byte aligned).
int sss_scratch(sss_ctx* ctx, size_t bytes, void** out);
int sss_counters(sss_ctx* ctx, size_t n, unsigned** out);
// Bounded-wait self-tests (a wait that nothing completes; sss_selftest_wait).
int sss_frame_barrier_selftest(sss_ctx* ctx, double limit_s, cudaStream_t s);
int sss_stream_barrier_selftest(sss_ctx* ctx, double limit_s, cudaStream_t s);

#define SSS_CUDA_TRY(ctx, call)                                   \
    do {                                                          \
        cudaError_t e__ = (call);                                 \
        if (e__ != cudaSuccess) return sss_cuda_err(ctx, e__, #call); \
    } while (0)

#define SSS_LAUNCH_CHECK(ctx, what)                               \
    do {                                                          \
        cudaError_t e__ = cudaGetLastError();                     \
        if (e__ != cudaSuccess) return sss_cuda_err(ctx, e__, what); \
    } while (0)

// ------------------------------------------------------------ device side

// Wall-clock limit of every spin on an mbarrier or flag (nanoseconds). A
// legitimate wait here is microseconds; the limit only turns a would-be hang
// into an SSS_ERR_TIMEOUT status.
#define SSS_WAIT_LIMIT_NS 2000000000ull

__device__ __forceinline__ uint64_t sss_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned sss_smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void sss_mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(sss_smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void sss_mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(sss_smem_addr(bar)), "r"(count) : "memory");
}

// Make mbarrier initialisation visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void sss_fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void sss_mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(sss_smem_addr(bar)), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar` (bytes must be
// a multiple of 16, both addresses 16-byte aligned).
__device__ __forceinline__ void sss_bulk_g2s(void* dst, const void* src, unsigned bytes,
                                             uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        :: "r"(sss_smem_addr(dst)), "l"(src), "r"(bytes), "r"(sss_smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool sss_mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(sss_smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`. Returns false (and records
// SSS_ERR_TIMEOUT in *status) if the phase did not complete within limit_ns.
__device__ __forceinline__ bool sss_mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                      int* status, uint64_t limit_ns = SSS_WAIT_LIMIT_NS) {
    if (sss_mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = sss_globaltimer();
    while (!sss_mbar_try_wait(bar, parity)) {
        if (sss_globaltimer() - t0 > limit_ns) {
            atomicExch(status, SSS_ERR_TIMEOUT);
            return false;
        }
    }
    return true;
}

// ------------------------------------------------------------- f64 kernels

// Gm * r2^(-3/2) in f64 from an f32 reciprocal-square-root seed.
//
// Method (Householder-type series refinement of 1/sqrt, e.g. Householder,
// "The Numerical Treatment of a Single Nonlinear Equation", 1970): with a
// seed c ~ r2^(-1/2) and e = 1 - r2*c^2, the exact value is
//   r2^(-3/2) = c^3 (1 - e)^(-3/2) = c^3 (1 + 3/2 e + 15/8 e^2 + 35/16 e^3 + ...).
// The seed is the hardware f32 approximation (rsqrt.approx.f32, |e| < 1e-6
// here), so the cubic remainder is < 3e-18 and the series is cut after e^2.
// c is an f32 value, hence c*c is exact in f64 and e carries one rounding.
// Cost: 7 f64 operations + one f32 MUFU op + two conversions.
__device__ __forceinline__ float sss_rsqrt_approx_f32(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ double sss_gm_rinv3_f64(double gm, double r2) {
    const float yf = sss_rsqrt_approx_f32(__double2float_rn(r2));
    const double c = (double)yf;
    const double c2 = c * c;                    // exact
    const double e = fma(-r2, c2, 1.0);         // 1 - r2 c^2
    const double p = fma(e, 1.875, 1.5);        // 3/2 + 15/8 e
    const double g = gm * c;
    const double g3 = g * c2;                   // Gm c^3
    return fma(g3, e * p, g3);                  // Gm c^3 (1 + e p)
}

// Same series with the seed's argument formed by integer operations instead
// of an f64->f32 conversion: the high word of r2 (sign, 11-bit exponent, 20
// mantissa bits) re-biased to an f32 bit pattern (mantissa truncated, |rel.
// error| < 2^-20), and the f32 result widened to f64 bit by bit. Valid for
// 2^-126 <= r2 < 2^128 (|e| < 1.3e-6, cubic remainder < 5e-18).
__device__ __forceinline__ double sss_gm_rinv3_f64_iseed(double gm, double r2) {
    const unsigned hi = (unsigned)__double2hiint(r2);
    const unsigned fb = (hi << 3) + 0x40000000u;          // exponent 1023 -> 127 bias
    const float yf = sss_rsqrt_approx_f32(__uint_as_float(fb));
    const unsigned yb = __float_as_uint(yf);
    const double c = __hiloint2double((int)((yb >> 3) + 0x38000000u), (int)(yb << 29));
    const double c2 = c * c;
    const double e = fma(-r2, c2, 1.0);
    const double p = fma(e, 1.875, 1.5);
    const double g = gm * c;
    const double g3 = g * c2;
    return fma(g3, e * p, g3);
}

// Same value from CUDA's own f64 rsqrt (kept as a selectable variant so the
// faster form can be chosen by measurement).
__device__ __forceinline__ double sss_gm_rinv3_cuda(double gm, double r2) {
    const double inv = rsqrt(r2);
    return ((gm * inv) * inv) * inv;
}

// f32 hypot, correctly rounded as the C library's hypotf (which NumPy calls for float32
// hypot): the squares of f32 values are exact in f64, their sum is rounded once, the square
// root once, then the result to f32.
__device__ __forceinline__ float sss_hypot_f32(float x, float y) {
    if (isinf(x) || isinf(y)) return __int_as_float(0x7F800000);
    const double xd = x, yd = y;
    return __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(xd, xd), __dmul_rn(yd, yd))));
}
