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

#include "devscan.cuh"

#include <algorithm>

namespace {

constexpr int K = 512;                 // LOD cells per axis (server.py LOD_ZELLEN)
constexpr int K2 = K * K;
constexpr int LEAVES = K2 / 128;       // 2048 pairwise-sum leaves
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

// tier per body: 0 culled out, 1 massive, 2 asteroid, 3 injected asteroid
__global__ void k_cull(const float* __restrict__ qx, const float* __restrict__ qy, const double* __restrict__ kill_t,
                       double t_cut, const unsigned char* __restrict__ is_ast,
                       const unsigned char* __restrict__ injected, long long n, Box b,
                       unsigned char* __restrict__ tier, unsigned long long* __restrict__ cnt4) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned char t = 0;
    if (kill_t[i] > t_cut && qx[i] >= b.x0 && qx[i] <= b.x1 && qy[i] >= b.y0 && qy[i] <= b.y1)
        t = !is_ast[i] ? 1 : (injected && injected[i] ? 3 : 2);
    tier[i] = t;
    if (t) atomicAdd(cnt4 + t, 1ull);
}

__device__ __forceinline__ int cell_of(float q, float o, float s) {
    const int c = (int)__fmul_rn(__fdiv_rn(__fsub_rn(q, o), s), (float)K);
    return min(max(c, 0), K - 1);
}

// counts of the bodies whose tier is in the mask (bit t = tier t)
__global__ void k_hist(const float* __restrict__ qx, const float* __restrict__ qy,
                       const unsigned char* __restrict__ tier, long long n, int mask, Box b,
                       int* __restrict__ counts) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !((mask >> tier[i]) & 1)) return;
    atomicAdd(counts + cell_of(qy[i], b.y0, b.sy) * K + cell_of(qx[i], b.x0, b.sx), 1);
}

__global__ void k_weights(const int* __restrict__ counts, double* __restrict__ w) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < K2) w[c] = counts[c] > 0 ? __dsqrt_rn((double)counts[c]) : 0.0;
}

// one pairwise-sum leaf of 128 cells of min(count, s w), s = (lo + hi) / 2
__global__ void k_leaf(const int* __restrict__ counts, const double* __restrict__ w,
                       const double* __restrict__ lohi, double* __restrict__ leaf) {
    const int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= LEAVES) return;
    const double s = __dmul_rn(0.5, __dadd_rn(lohi[0], lohi[1]));
    const int base = L * 128;
    double r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = fmin((double)counts[base + j], __dmul_rn(s, w[base + j]));
    for (int i = 8; i < 128; i += 8)
#pragma unroll
        for (int j = 0; j < 8; ++j)
            r[j] = __dadd_rn(r[j], fmin((double)counts[base + i + j], __dmul_rn(s, w[base + i + j])));
    leaf[L] = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                        __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
}

// pairwise levels over the 2048 leaves (left + right), then the bisection step
__global__ void __launch_bounds__(1024) k_tree(const double* __restrict__ leaf, double budget,
                                              double* __restrict__ lohi) {
    __shared__ double s[LEAVES];
    for (int i = threadIdx.x; i < LEAVES; i += blockDim.x) s[i] = leaf[i];
    __syncthreads();
    for (int m = LEAVES / 2; m >= 1; m >>= 1) {
        double v = 0.0;
        if ((int)threadIdx.x < m) v = __dadd_rn(s[2 * threadIdx.x], s[2 * threadIdx.x + 1]);
        __syncthreads();
        if ((int)threadIdx.x < m) s[threadIdx.x] = v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double sm = __dmul_rn(0.5, __dadd_rn(lohi[0], lohi[1]));
        if (s[0] > budget) lohi[1] = sm;
        else lohi[0] = sm;
    }
}

__global__ void k_rates(const int* __restrict__ counts, const double* __restrict__ w, const double* __restrict__ lohi,
                        double* __restrict__ rate) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K2) return;
    const double lo = lohi[0];
    rate[c] = counts[c] > 0 ? __ddiv_rn(fmin((double)counts[c], __dmul_rn(lo, w[c])), (double)counts[c]) : 0.0;
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

// keep decision of the bodies of the masked tiers; keep[i] = 1, count kept
__global__ void k_keep(const float* __restrict__ qx, const float* __restrict__ qy,
                       const unsigned char* __restrict__ tier, long long n, int mask, Box b,
                       const double* __restrict__ rate, unsigned char* __restrict__ keep,
                       unsigned long long* __restrict__ kept) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !((mask >> tier[i]) & 1)) return;
    const float fx = frac_coord(qx[i], b.x0, b.sx), fy = frac_coord(qy[i], b.y0, b.sy);
    const int ix = (int)floorf(fx), iy = (int)floorf(fy);
    const int ix1 = min(ix + 1, K - 1), iy1 = min(iy + 1, K - 1);
    const double tx = __dsub_rn((double)fx, (double)ix), ty = __dsub_rn((double)fy, (double)iy);
    const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
    double rp = __dmul_rn(__dmul_rn(rate[iy * K + ix], ux), uy);
    rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(rate[iy * K + ix1], tx), uy));
    rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(rate[iy1 * K + ix], ux), ty));
    rp = __dadd_rn(rp, __dmul_rn(__dmul_rn(rate[iy1 * K + ix1], tx), ty));
    if (index_hash((unsigned long long)i) < rp) {
        keep[i] = 1;
        atomicAdd(kept, 1ull);
    }
}

// keep[i] = 1 for every body of the masked tiers (a tier under its budget)
__global__ void k_keep_all(const unsigned char* __restrict__ tier, long long n, int mask,
                           unsigned char* __restrict__ keep) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && ((mask >> tier[i]) & 1)) keep[i] = 1;
}

__global__ void k_keep_flags(const unsigned char* __restrict__ keep, long long n, long long* __restrict__ f) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = keep[i];
}

__device__ __forceinline__ unsigned short quant(float q, float o, float s) {
    const float v = __fmul_rn(__fdiv_rn(__fsub_rn(q, o), s), 65535.0f);
    return (unsigned short)fminf(fmaxf(v, 0.0f), 65535.0f);
}

__global__ void k_emit(const float* __restrict__ qx, const float* __restrict__ qy, const long long* __restrict__ f,
                       const long long* __restrict__ pos, long long n, Box b, unsigned* __restrict__ sel,
                       unsigned short* __restrict__ ox, unsigned short* __restrict__ oy) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !f[i]) return;
    const long long q = pos[i];
    sel[q] = (unsigned)i;
    ox[q] = quant(qx[i], b.x0, b.sx);
    oy[q] = quant(qy[i], b.y0, b.sy);
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

struct Work {
    float *qx, *qy;
    unsigned char *tier, *keep;
    int* counts;
    double *w, *rate, *leaf, *lohi;
    unsigned long long* cnt;           // [0..3] tier counts, [4] kept
    long long *flags, *pos, *scan;
};

// density filter of the masked tiers with `budget` points (the reference's
// _dichte_filter); returns the number kept (all of them when under budget)
int density_filter(sss_ctx* ctx, const Work& W, long long n, int mask, long long size, long long budget, Box b,
                   cudaStream_t st, long long* kept) {
    if (size <= budget) {
        k_keep_all<<<nb(n), 256, 0, st>>>(W.tier, n, mask, W.keep);
        SSS_LAUNCH_CHECK(ctx, "k_keep_all");
        *kept = size;
        return SSS_OK;
    }
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(W.counts, 0, K2 * sizeof(int), st));
    k_hist<<<nb(n), 256, 0, st>>>(W.qx, W.qy, W.tier, n, mask, b, W.counts);
    SSS_LAUNCH_CHECK(ctx, "k_hist");
    k_weights<<<K2 / 256, 256, 0, st>>>(W.counts, W.w);
    const double lohi0[2] = {0.0, (double)budget};
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(W.lohi, lohi0, sizeof(lohi0), cudaMemcpyHostToDevice, st));
    for (int it = 0; it < 40; ++it) {
        k_leaf<<<LEAVES / 256, 256, 0, st>>>(W.counts, W.w, W.lohi, W.leaf);
        k_tree<<<1, 1024, 0, st>>>(W.leaf, (double)budget, W.lohi);
    }
    k_rates<<<K2 / 256, 256, 0, st>>>(W.counts, W.w, W.lohi, W.rate);
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(W.cnt + 4, 0, 8, st));
    k_keep<<<nb(n), 256, 0, st>>>(W.qx, W.qy, W.tier, n, mask, b, W.rate, W.keep, W.cnt + 4);
    SSS_LAUNCH_CHECK(ctx, "k_keep");
    unsigned long long k = 0;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&k, W.cnt + 4, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    *kept = (long long)k;
    return SSS_OK;
}

int make_work(sss_ctx* ctx, long long n, Work* W) {
    size_t off = 0;
    const size_t o_qx = off; off += al((size_t)n * 4);
    const size_t o_qy = off; off += al((size_t)n * 4);
    const size_t o_tier = off; off += al((size_t)n);
    const size_t o_keep = off; off += al((size_t)n);
    const size_t o_cnts = off; off += al((size_t)K2 * 4);
    const size_t o_w = off; off += al((size_t)K2 * 8);
    const size_t o_rate = off; off += al((size_t)K2 * 8);
    const size_t o_leaf = off; off += al((size_t)LEAVES * 8);
    const size_t o_lohi = off; off += al(16);
    const size_t o_cnt = off; off += al(8 * 8);
    const size_t o_flags = off; off += al((size_t)n * 8);
    const size_t o_pos = off; off += al((size_t)n * 8);
    const size_t o_scan = off; off += al(sss_dev::scan_scratch(n) * 8);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* p = (char*)scr;
    W->qx = (float*)(p + o_qx);
    W->qy = (float*)(p + o_qy);
    W->tier = (unsigned char*)(p + o_tier);
    W->keep = (unsigned char*)(p + o_keep);
    W->counts = (int*)(p + o_cnts);
    W->w = (double*)(p + o_w);
    W->rate = (double*)(p + o_rate);
    W->leaf = (double*)(p + o_leaf);
    W->lohi = (double*)(p + o_lohi);
    W->cnt = (unsigned long long*)(p + o_cnt);
    W->flags = (long long*)(p + o_flags);
    W->pos = (long long*)(p + o_pos);
    W->scan = (long long*)(p + o_scan);
    return SSS_OK;
}

}  // namespace

extern "C" int sss_stream_minmax(sss_ctx* ctx, int64_t n, const float* x, const float* y, int log_zoom, float* out4,
                                 void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (n < 1 || !x || !y || !out4) return sss_set_err(ctx, SSS_ERR_ARG, "minmax: empty or NULL input");
    cudaStream_t st = (cudaStream_t)stream;
    Work W;
    int rc = make_work(ctx, n, &W);
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
    float* part = (float*)W.w;                   // 4 floats per block
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

extern "C" int sss_stream_sample(sss_ctx* ctx, int64_t n, const float* x, const float* y, const double* kill_t,
                                 double t_cut, const unsigned char* is_ast, const unsigned char* injected,
                                 const double* box, int log_zoom, int64_t budget, unsigned* sel, uint16_t* qx_out,
                                 uint16_t* qy_out, int64_t* n_sel, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!n_sel || !box) return sss_set_err(ctx, SSS_ERR_ARG, "NULL box or count");
    *n_sel = 0;
    if (n < 0 || budget < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n == 0) return SSS_OK;
    if (!x || !y || !kill_t || !is_ast || !sel || !qx_out || !qy_out)
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    cudaStream_t st = (cudaStream_t)stream;
    Work W;
    int rc = make_work(ctx, n, &W);
    if (rc) return rc;
    Box b;
    b.x0 = (float)box[0];
    b.y0 = (float)box[1];
    b.sx = (float)box[2];
    b.sy = (float)box[3];
    b.x1 = (float)(box[0] + box[2]);
    b.y1 = (float)(box[1] + box[3]);
    const float* qx = x;
    const float* qy = y;
    if (log_zoom) {
        k_disp<<<nb(n), 256, 0, st>>>(x, y, n, W.qx, W.qy);
        SSS_LAUNCH_CHECK(ctx, "k_disp");
        qx = W.qx;
        qy = W.qy;
    }
    W.qx = (float*)qx;
    W.qy = (float*)qy;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(W.cnt, 0, 8 * 8, st));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(W.keep, 0, (size_t)n, st));
    k_cull<<<nb(n), 256, 0, st>>>(qx, qy, kill_t, t_cut, is_ast, injected, n, b, W.tier, W.cnt);
    SSS_LAUNCH_CHECK(ctx, "k_cull");
    unsigned long long c[4] = {0, 0, 0, 0};
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(c, W.cnt, sizeof(c), cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    const long long mm = (long long)c[1], ma = (long long)c[2], mi = (long long)c[3];
    const long long m = mm + ma + mi;
    const int T_ALL = (1 << 1) | (1 << 2) | (1 << 3), T_MASS = 1 << 1, T_AST = (1 << 2) | (1 << 3);
    long long kept = 0;
    if (m <= budget) {
        k_keep_all<<<nb(n), 256, 0, st>>>(W.tier, n, T_ALL, W.keep);
        SSS_LAUNCH_CHECK(ctx, "k_keep_all");
    } else {
        long long rest = budget - mm;
        if (rest <= 0) {
            if (mm > 200 && m > mm) {
                // many massive bodies (a self-gravity cloud): they get half the budget, thinned
                const long long m_budget = std::max<long long>(1, (long long)((double)budget * 0.5));
                rc = density_filter(ctx, W, n, T_MASS, mm, m_budget, b, st, &kept);
                if (rc) return rc;
                rest = budget - kept;
                if (rest > 0 && ma + mi > 0) {
                    rc = density_filter(ctx, W, n, T_AST, ma + mi, rest, b, st, &kept);
                    if (rc) return rc;
                }
            } else {
                k_keep_all<<<nb(n), 256, 0, st>>>(W.tier, n, T_MASS, W.keep);
                SSS_LAUNCH_CHECK(ctx, "k_keep_all");
            }
        } else {
            k_keep_all<<<nb(n), 256, 0, st>>>(W.tier, n, T_MASS, W.keep);
            SSS_LAUNCH_CHECK(ctx, "k_keep_all");
            const long long sizes[2] = {ma, mi};
            const int masks[2] = {1 << 2, 1 << 3};
            for (int q = 0; q < 2; ++q) {
                if (rest <= 0 || sizes[q] == 0) continue;
                rc = density_filter(ctx, W, n, masks[q], sizes[q], rest, b, st, &kept);
                if (rc) return rc;
                rest -= kept;
            }
        }
    }
    k_keep_flags<<<nb(n), 256, 0, st>>>(W.keep, n, W.flags);
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(W.flags, W.pos, n, W.scan, st));
    k_emit<<<nb(n), 256, 0, st>>>(qx, qy, W.flags, W.pos, n, b, sel, qx_out, qy_out);
    SSS_LAUNCH_CHECK(ctx, "k_emit");
    long long tot = 0;
    const long long tiles = (n + sss_dev::SCAN_TILE - 1) / sss_dev::SCAN_TILE;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(&tot, W.scan + tiles, 8, cudaMemcpyDeviceToHost, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    *n_sel = tot;
    return SSS_OK;
}
