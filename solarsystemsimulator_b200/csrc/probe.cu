// Throughput probe: the FP64 / FP32 SIMT FMA peaks the all-pairs kernels are
// measured against (the driver-measured peaks cover only HBM copy and bf16
// tensor GEMM), and the rate of the f32 reciprocal square root (the special
// function unit) that bounds the mixed-precision pair loop. Diagnostic entry
// point, no reference counterpart.
#include "sss_internal.cuh"

namespace {

constexpr int CHAINS = 8;

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(T* out, int iters, T a, T b) {
    T x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// packed f32x2 FMA (sm_100a): two f32 lanes per thread per instruction
__global__ void __launch_bounds__(256) k_fma_chain_x2(float* out, int iters, float a, float b) {
    unsigned long long x[CHAINS];
    unsigned long long av, bv;
    asm("mov.b64 %0, {%1, %1};" : "=l"(av) : "f"(a));
    asm("mov.b64 %0, {%1, %1};" : "=l"(bv) : "f"(b));
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) {
        const float v0 = (float)(threadIdx.x + c) * 1e-3f, v1 = v0 + 0.5f;
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[c]) : "f"(v0), "f"(v1));
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c)
            asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[c]) : "l"(av), "l"(bv));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[c]));
        s += lo + hi;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// chains of rsqrt.approx.f32: one special-function operation per step
__global__ void __launch_bounds__(256) k_rsqrt_chain(float* out, int iters) {
    float x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = 1.5f + (float)(threadIdx.x + c) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) x[c] = sss_rsqrt_approx_f32(x[c]) + 1.0f;
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int sss_probe_fma(sss_ctx* ctx, int kind, int iters, double* tflops) {
    if (!ctx || !tflops) return SSS_ERR_ARG;
    if (kind < 0 || kind > 3)
        return sss_set_err(ctx, SSS_ERR_ARG, "kind must be 0 (f64), 1 (f32), 2 (f32x2), 3 (f32 rsqrt)");
    if (iters < 1) return sss_set_err(ctx, SSS_ERR_ARG, "iters must be >= 1");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    const int blocks = ctx->num_sms * 8, threads = 256;
    void* out = nullptr;
    int rc = sss_scratch(ctx, (size_t)blocks * threads * sizeof(double), &out);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    SSS_CUDA_TRY(ctx, cudaEventCreate(&e0));
    SSS_CUDA_TRY(ctx, cudaEventCreate(&e1));
    float best_ms = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {  // first launch is a warm-up
        cudaEventRecord(e0);
        if (kind == 0) k_fma_chain<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
        else if (kind == 1) k_fma_chain<float><<<blocks, threads>>>((float*)out, iters, 0.9999f, 1e-4f);
        else if (kind == 2) k_fma_chain_x2<<<blocks, threads>>>((float*)out, iters, 0.9999f, 1e-4f);
        else k_rsqrt_chain<<<blocks, threads>>>((float*)out, iters);
        cudaEventRecord(e1);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return sss_cuda_err(ctx, e, "probe kernel");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_ms) best_ms = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // FMA kinds: 2 flops per lane and FMA; rsqrt: 1 operation per step
    const double per_step = (kind == 2) ? 4.0 : (kind == 3 ? 1.0 : 2.0);
    const double flops = per_step * CHAINS * (double)iters * blocks * threads;
    *tflops = flops / (best_ms * 1e-3) / 1e12;
    return SSS_OK;
}

namespace {

// Self-test of the mbarrier wait the bulk-copy and tensor-core kernels use:
// an mbarrier that expects two arrivals gets one, so the wait for its phase
// runs out after limit_ns and records SSS_ERR_TIMEOUT.
__global__ void k_mbar_selftest(uint64_t limit_ns, int* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        sss_mbar_init(&bar, 2);
        sss_fence_mbar_init();
        sss_mbar_arrive(&bar);
        sss_mbar_wait_bounded(&bar, 0, status, limit_ns);
    }
}

}  // namespace

extern "C" int sss_selftest_wait(sss_ctx* ctx, int which, double limit_s, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (which < 0 || which > 2) return sss_set_err(ctx, SSS_ERR_ARG, "which must be 0, 1 or 2");
    if (!(limit_s > 0.0 && limit_s <= 10.0)) return sss_set_err(ctx, SSS_ERR_ARG, "limit_s must be in (0, 10]");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (which == 1) return sss_frame_barrier_selftest(ctx, limit_s, s);
    if (which == 2) return sss_stream_barrier_selftest(ctx, limit_s, s);
    k_mbar_selftest<<<1, 32, 0, s>>>((uint64_t)(limit_s * 1e9), ctx->d_status);
    SSS_LAUNCH_CHECK(ctx, "k_mbar_selftest");
    return SSS_OK;
}
