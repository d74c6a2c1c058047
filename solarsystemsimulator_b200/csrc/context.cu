// Context, error and scratch management of libsss (the C ABI in include/sss.h).
#include "sss_internal.cuh"

#include <stdlib.h>

int sss_set_err(sss_ctx* ctx, int code, const char* fmt, ...) {
    if (ctx) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int sss_cuda_err(sss_ctx* ctx, cudaError_t e, const char* what) {
    return sss_set_err(ctx, SSS_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

int sss_scratch(sss_ctx* ctx, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~(size_t)255;
    if (bytes > ctx->scratch_bytes) {
        if (ctx->scratch) {
            // the previous scratch may still be read by queued kernels
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaDeviceSynchronize (scratch grow)");
            cudaFree(ctx->scratch);
            ctx->scratch = nullptr;
            ctx->scratch_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&ctx->scratch, bytes);
        if (e != cudaSuccess) {
            ctx->scratch = nullptr;
            return sss_cuda_err(ctx, e, "cudaMalloc (scratch)");
        }
        ctx->scratch_bytes = bytes;
    }
    *out = ctx->scratch;
    return SSS_OK;
}

int sss_counters(sss_ctx* ctx, size_t n, unsigned** out) {
    if (n > ctx->n_counters) {
        if (ctx->d_counters) {
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaDeviceSynchronize (counters grow)");
            cudaFree(ctx->d_counters);
            ctx->d_counters = nullptr;
            ctx->n_counters = 0;
        }
        size_t cap = n < 4096 ? 4096 : n;
        cudaError_t e = cudaMalloc(&ctx->d_counters, cap * sizeof(unsigned));
        if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaMalloc (counters)");
        e = cudaMemset(ctx->d_counters, 0, cap * sizeof(unsigned));
        if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaMemset (counters)");
        ctx->n_counters = cap;
    }
    *out = ctx->d_counters;
    return SSS_OK;
}

extern "C" int sss_abi_version(void) { return SSS_ABI_VERSION; }

extern "C" int sss_create(int device, sss_ctx** out) {
    if (!out) return SSS_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return SSS_ERR_CUDA;
    if (device < 0 || device >= n) return SSS_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SSS_ERR_CUDA;
    sss_ctx* c = (sss_ctx*)calloc(1, sizeof(sss_ctx));
    if (!c) return SSS_ERR_CUDA;
    c->device = device;
    if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        free(c);
        return SSS_ERR_CUDA;
    }
    if (cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess || cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess) {
        free(c);
        return SSS_ERR_CUDA;
    }
    snprintf(c->err, sizeof(c->err), "no error");
    *out = c;
    return SSS_OK;
}

extern "C" void sss_destroy(sss_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    sss_bp_graph_free(ctx->bp_graph);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    if (ctx->d_status) cudaFree(ctx->d_status);
    free(ctx);
}

extern "C" const char* sss_last_error(const sss_ctx* ctx) {
    return ctx ? ctx->err : "NULL context";
}

extern "C" int sss_num_sms(const sss_ctx* ctx) { return ctx ? ctx->num_sms : 0; }

extern "C" int sss_device_status(sss_ctx* ctx, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaStreamSynchronize");
    int h = 0;
    e = cudaMemcpy(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaMemcpy (status)");
    if (h != 0) {
        cudaMemset(ctx->d_status, 0, sizeof(int));
        return sss_set_err(ctx, h, h == SSS_ERR_GUARD ? "device reported status %d (a step guard ran out)"
                                                      : "device reported status %d (a bounded wait timed out)", h);
    }
    return SSS_OK;
}
