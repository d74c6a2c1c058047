// The film producer's ring slots written on the device (reference
// backend/film_producer.py:79-123 slot_bytes / schreibe_slot) and the
// self-gravity row reorder into the client's body order (:1245-1261).
//
// A slot is x|y f32 (8n bytes) | u32 count | u32 indices (a field of sub_max
// entries) | f32 sub-sample chains (nh, mSub, 2): the hot asteroids of the
// sample (the frame kernel recorded a gap-free chain of m_sub sub-samples
// for them) in ascending original index, at most sub_max of them, each
// chain stored body by body. The frame kernel keeps the sub-samples as
// [m_sub][dim][n_ast]; the slot kernel transposes them while compacting.
// Entries of the index field and chains beyond the count are left as they
// were, as the reference leaves them.

#include "devscan.cuh"

namespace {

__global__ void k_hot_flags(const unsigned char* __restrict__ sub_n, long long n_ast, int m_sub,
                            long long* __restrict__ flags) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n_ast) flags[s] = sub_n[s] == m_sub ? 1 : 0;
}

__global__ void k_hot_write(const long long* __restrict__ flags, const long long* __restrict__ pos,
                            const float* __restrict__ sub_pos, const long long* __restrict__ a_idx, long long n_ast,
                            int m_sub, long long sub_max, unsigned* __restrict__ idx_field,
                            float* __restrict__ chains) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_ast || !flags[s]) return;
    const long long q = pos[s];
    if (q >= sub_max) return;                // overflow: the lowest indices are kept
    idx_field[q] = (unsigned)a_idx[s];
    // sub_pos[j][c][s] (component c = 0, 1 of dim) -> chains[q][j][c]
    const long long plane = n_ast;           // stride of one component
    for (int j = 0; j < m_sub; ++j) {
        chains[(q * m_sub + j) * 2] = sub_pos[((long long)j * 2 + 0) * plane + s];
        chains[(q * m_sub + j) * 2 + 1] = sub_pos[((long long)j * 2 + 1) * plane + s];
    }
}

// same for dim == 3 layouts ([m_sub][3][n_ast]): components 0 and 1 only
__global__ void k_hot_write3(const long long* __restrict__ flags, const long long* __restrict__ pos,
                             const float* __restrict__ sub_pos, const long long* __restrict__ a_idx,
                             long long n_ast, int m_sub, long long sub_max, unsigned* __restrict__ idx_field,
                             float* __restrict__ chains) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_ast || !flags[s]) return;
    const long long q = pos[s];
    if (q >= sub_max) return;
    idx_field[q] = (unsigned)a_idx[s];
    for (int j = 0; j < m_sub; ++j) {
        chains[(q * m_sub + j) * 2] = sub_pos[((long long)j * 3 + 0) * n_ast + s];
        chains[(q * m_sub + j) * 2 + 1] = sub_pos[((long long)j * 3 + 1) * n_ast + s];
    }
}

__global__ void k_count(const long long* __restrict__ scan_total, long long sub_max, unsigned* __restrict__ count) {
    const long long t = *scan_total;
    *count = (unsigned)(t < sub_max ? t : sub_max);
}

// rows [K][4 nm + 2 nt] (masses x|y|vx|vy, tracers x|y) -> out [K][4n]
__global__ void k_reorder(const float* __restrict__ rows, int K, const long long* __restrict__ sg_m, long long nm,
                          const long long* __restrict__ sg_t, long long nt, long long n, float* __restrict__ out) {
    const long long w = 4 * nm + 2 * nt;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)K * w) return;
    const long long k = t / w, e = t % w;
    long long dst;
    if (e < 4 * nm) {
        const long long c = e / nm, i = e % nm;
        dst = c * n + sg_m[i];
    } else {
        const long long e2 = e - 4 * nm;
        const long long c = e2 / nt, i = e2 % nt;
        dst = c * n + sg_t[i];
    }
    out[k * 4 * n + dst] = rows[t];
}

size_t al(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

extern "C" int sss_ring_slot(sss_ctx* ctx, const float* row, int64_t n, const float* sub_pos,
                             const unsigned char* sub_n, const int64_t* a_idx, int64_t n_ast, int m_sub, int dim,
                             int64_t sub_max, unsigned char* slot, int64_t* n_hot, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!n_hot) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count pointer");
    *n_hot = 0;
    if (n < 0 || n_ast < 0 || sub_max < 0 || m_sub < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n_ast > n) return sss_set_err(ctx, SSS_ERR_ARG, "more asteroids than bodies");
    if (!slot || (n > 0 && !row)) return sss_set_err(ctx, SSS_ERR_ARG, "NULL row or slot");
    if (dim != 2 && dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3");
    cudaStream_t st = (cudaStream_t)stream;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(slot, row, (size_t)8 * n, cudaMemcpyDeviceToDevice, st));
    unsigned* count = (unsigned*)(slot + 8 * n);
    const bool subs = sub_pos && sub_n && a_idx && sub_max > 0 && m_sub > 0 && n_ast > 0;
    if (!subs) {
        SSS_CUDA_TRY(ctx, cudaMemsetAsync(count, 0, 4, st));
        SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        return SSS_OK;
    }
    void* scr = nullptr;
    const size_t o_flags = 0, o_pos = al((size_t)n_ast * 8), o_scan = o_pos + al((size_t)n_ast * 8);
    int rc = sss_scratch(ctx, o_scan + al(sss_dev::scan_scratch(n_ast) * 8), &scr);
    if (rc) return rc;
    long long* flags = (long long*)((char*)scr + o_flags);
    long long* pos = (long long*)((char*)scr + o_pos);
    long long* scan = (long long*)((char*)scr + o_scan);
    const unsigned nb = (unsigned)((n_ast + 255) / 256);
    k_hot_flags<<<nb, 256, 0, st>>>(sub_n, n_ast, m_sub, flags);
    SSS_LAUNCH_CHECK(ctx, "k_hot_flags");
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(flags, pos, n_ast, scan, st, ctx->d_status));
    const long long tiles = (n_ast + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    k_count<<<1, 1, 0, st>>>(scan + tiles, sub_max, count);
    SSS_LAUNCH_CHECK(ctx, "k_count");
    unsigned* idx_field = count + 1;
    float* chains = (float*)(idx_field + sub_max);
    if (dim == 2)
        k_hot_write<<<nb, 256, 0, st>>>(flags, pos, sub_pos, (const long long*)a_idx, n_ast, m_sub, sub_max,
                                        idx_field, chains);
    else
        k_hot_write3<<<nb, 256, 0, st>>>(flags, pos, sub_pos, (const long long*)a_idx, n_ast, m_sub, sub_max,
                                         idx_field, chains);
    SSS_LAUNCH_CHECK(ctx, "k_hot_write");
    long long total = 0;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&total, scan + tiles, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    *n_hot = total;
    return SSS_OK;
}

extern "C" int sss_ring_reorder(sss_ctx* ctx, const float* rows, int K, const int64_t* sg_m, int64_t nm,
                                const int64_t* sg_t, int64_t nt, int64_t n, float* out, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (K < 0 || nm < 0 || nt < 0 || n < 0 || nm + nt > n) return sss_set_err(ctx, SSS_ERR_ARG, "bad sizes");
    if (K == 0 || n == 0) return SSS_OK;
    if (!rows || !out || (nm > 0 && !sg_m) || (nt > 0 && !sg_t)) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    cudaStream_t st = (cudaStream_t)stream;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(out, 0, (size_t)K * 4 * n * sizeof(float), st));
    const long long tot = (long long)K * (4 * nm + 2 * nt);
    if (tot == 0) return SSS_OK;
    k_reorder<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(rows, K, (const long long*)sg_m, nm,
                                                             (const long long*)sg_t, nt, n, out);
    SSS_LAUNCH_CHECK(ctx, "k_reorder");
    return SSS_OK;
}
