// f64 Ewald direct sum: the exact periodic force that judges the mesh forces
// and supplies the training targets of the learned correction.
//
// a_i = -G sum_j m_j d_ij [ (erfc(x) + 2 x / sqrt(pi) e^{-x^2}) / r^3   (r < r_cut, x = alpha r)
//                           + (r^2 + eps2)^{-3/2} - r^{-3} ]        (every pair)
//       -G sum_{h in half space} coef_h k_h [ sin(k.x_i) C_h - cos(k.x_i) S_h ]
// over the nearest image d_ij of every source, with (C_h, S_h) =
// sum_j m_j (cos, sin)(k_h . x_j), k = 2 pi h / box. The erfc term is the
// real-space part of the periodic Newtonian force, the reciprocal sum holds
// its long-range erf part of every image (Hernquist, Bouchet & Suto 1991),
// and the Plummer correction turns the nearest image's 1/r^2 into the
// softened force for every pair, so the result does not depend on alpha.
// Close pairs (r^2 < max(1000 eps2, (0.5/alpha)^2)) use the combined form
// (-erf(x) + 2 x / sqrt(pi) e^{-x^2}) / r^3 + (r^2 + eps2)^{-3/2}, far pairs
// the correction as the series of (1 + u)^{-3/2} - 1 in u = eps2 / r^2
// (u < 1e-3 there), so neither form cancels two large 1/r^3 terms.
//
// Kernels: k_ewald_sk builds the structure factors (one thread per k
// vector, a CTA walks a slice of the particles whose e^{i 2 pi h x} power
// tables it stages in shared memory, so each term costs two complex
// products); k_ewald_real is the target x source real-space sum (a warp
// per target over the sources in Morton order, the erfc factor from a
// table; the source list split into chunks for parallelism, partials added
// in chunk order); k_ewald_final adds the partials and the reciprocal part
// per target. Deterministic.

#include "pm3d.cuh"
#include "devscan.cuh"

#include <algorithm>
#include <cmath>

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr int SK_NT = 256;      // k vectors per CTA
constexpr int SK_TILE = 32;     // particles per staged table
constexpr int RS_WARPS = 8;     // targets per CTA of the real-space sum (a warp each)
constexpr int RS_NT = RS_WARPS * 32;
constexpr int MORTON_BITS = 7;  // 128^3 cells for the source order

__global__ void __launch_bounds__(SK_NT) k_ewald_sk(const Pm3Parts s, double inv_box, const int* __restrict__ hvec,
                                                    int nk, int hmax, long long per_chunk,
                                                    double2* __restrict__ part) {
    extern __shared__ double2 tab[];            // [SK_TILE][3][hmax + 1]
    __shared__ double s_m[SK_TILE];
    const int H = hmax + 1;
    const int kk = blockIdx.x * SK_NT + threadIdx.x;
    int hx = 0, hy = 0, hz = 0;
    bool use = false;
    if (kk < nk) {
        hx = hvec[3 * kk];
        hy = hvec[3 * kk + 1];
        hz = hvec[3 * kk + 2];
        use = hx >= 0 && hx <= hmax && abs(hy) <= hmax && abs(hz) <= hmax;
        if (!use) hx = hy = hz = 0;     // table index stays in range; result discarded
    }
    const int ay = abs(hy), az = abs(hz);
    const double sy = hy < 0 ? -1.0 : 1.0, sz = hz < 0 ? -1.0 : 1.0;
    const long long p0 = (long long)blockIdx.y * per_chunk;
    const long long p1 = min(s.n, p0 + per_chunk);
    double C = 0.0, S = 0.0;
    for (long long q0 = p0; q0 < p1; q0 += SK_TILE) {
        const int cnt = (int)min((long long)SK_TILE, p1 - q0);
        __syncthreads();
        if (threadIdx.x < 3 * SK_TILE) {
            const int q = threadIdx.x / 3, c = threadIdx.x % 3;
            double2* row = tab + (q * 3 + c) * H;
            if (q < cnt) {
                double sn, cs;
                sincospi(2.0 * s.x[c][q0 + q] * inv_box, &sn, &cs);
                double re = 1.0, im = 0.0;
                row[0] = make_double2(1.0, 0.0);
                for (int h = 1; h <= hmax; ++h) {
                    const double nr = re * cs - im * sn;
                    const double ni = re * sn + im * cs;
                    re = nr;
                    im = ni;
                    row[h] = make_double2(re, im);
                }
                if (c == 0) s_m[q] = s.m ? s.m[q0 + q] : s.mass_const;
            }
        }
        __syncthreads();
        for (int q = 0; q < cnt; ++q) {
            const double2 ex = tab[(q * 3 + 0) * H + hx];
            const double2 ey = tab[(q * 3 + 1) * H + ay];
            const double2 ez = tab[(q * 3 + 2) * H + az];
            const double eyi = sy * ey.y, ezi = sz * ez.y;
            const double xr = ex.x * ey.x - ex.y * eyi;
            const double xi = ex.x * eyi + ex.y * ey.x;
            const double m = s_m[q];
            C += m * (xr * ez.x - xi * ezi);
            S += m * (xr * ezi + xi * ez.x);
        }
    }
    if (kk < nk) part[(long long)blockIdx.y * nk + kk] = use ? make_double2(C, S) : make_double2(0.0, 0.0);
}

__global__ void k_ewald_sk_reduce(const double2* __restrict__ part, int nk, int chunks, double* __restrict__ sc) {
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    if (kk >= nk) return;
    double C = 0.0, S = 0.0;
    for (int c = 0; c < chunks; ++c) {
        const double2 v = part[(long long)c * nk + kk];
        C += v.x;
        S += v.y;
    }
    sc[2 * kk] = C;
    sc[2 * kk + 1] = S;
}

struct Targets {
    const double* t[3];
    const long long* self;
    long long n;
};

// g(x) = erfc(x) + 2 x e^{-x^2} / sqrt(pi), the real-space factor of the
// Ewald force, tabulated on [0, G_XMAX] as quintic Taylor pieces about the
// centres of G_NI intervals. Its derivatives are closed forms: g'(x) =
// -(4 / sqrt(pi)) x^2 e^{-x^2}, and d^j/dx^j (x^2 e^{-x^2}) = e^{-x^2} q_j(x)
// with q_0 = x^2, q_{j+1} = q_j' - 2 x q_j. The centre values use the C
// library's erfc and exp; over [0, 6] the pieces stay within 6e-16 of g
// (absolute; g(0) = 1), with the truncation of the series near 1e-17.
constexpr int G_NI = 1024, G_DEG = 5;
constexpr double G_XMAX = 6.0;
constexpr double G_H = G_XMAX / G_NI;
__device__ double g_gtab[G_NI * (G_DEG + 1)];

void build_gtab(double* tab) {
    const double sp = 1.1283791670955126;   // 2 / sqrt(pi)
    // q_j as coefficient lists (degree j + 2)
    double q[G_DEG][G_DEG + 3] = {};
    q[0][2] = 1.0;
    for (int j = 0; j + 1 < G_DEG; ++j) {
        for (int e = 0; e < G_DEG + 3; ++e) {
            double v = 0.0;
            if (e + 1 < G_DEG + 3) v += (e + 1) * q[j][e + 1];          // q_j'
            if (e >= 1) v -= 2.0 * q[j][e - 1];                          // -2 x q_j
            q[j + 1][e] = v;
        }
    }
    for (int k = 0; k < G_NI; ++k) {
        const double c = (k + 0.5) * G_H;
        const double ex = std::exp(-c * c);
        double* a = tab + k * (G_DEG + 1);
        a[0] = std::erfc(c) + sp * c * ex;
        double fact = 1.0;
        for (int j = 0; j < G_DEG; ++j) {
            double qv = 0.0;
            for (int e = G_DEG + 2; e >= 0; --e) qv = qv * c + q[j][e];
            fact *= (j + 1);
            a[j + 1] = -2.0 * sp * ex * qv / fact;
        }
    }
}

// upload the table once per device
int ensure_gtab(sss_ctx* ctx, cudaStream_t st) {
    static bool done[64];
    static double host[G_NI * (G_DEG + 1)];
    static bool built = false;
    const int dev = ctx->device;
    if (dev >= 0 && dev < 64 && done[dev]) return SSS_OK;
    if (!built) {
        build_gtab(host);
        built = true;
    }
    SSS_CUDA_TRY(ctx, cudaMemcpyToSymbolAsync(g_gtab, host, sizeof(host), 0, cudaMemcpyHostToDevice, st));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (dev >= 0 && dev < 64) done[dev] = true;
    return SSS_OK;
}

__device__ __forceinline__ double g_of(double x) {
    const int k = min((int)(x * (1.0 / G_H)), G_NI - 1);
    const double d = x - (k + 0.5) * G_H;
    const double2* a = (const double2*)(g_gtab + k * (G_DEG + 1));
    const double2 a01 = __ldg(a), a23 = __ldg(a + 1), a45 = __ldg(a + 2);
    return a01.x + d * (a01.y + d * (a23.x + d * (a23.y + d * (a45.x + d * a45.y))));
}

// the factor f(r) of one pair, a = -G m f d (see the file comment). The
// powers of r come from one reciprocal square root (CUDA's double rsqrt,
// 1 ulp); the erfc part from the table (alpha r_cut <= G_XMAX).
__device__ __forceinline__ double ewald_pair(double r2, double alpha, double eps2, double rc2, double small2) {
    const double sp = 1.1283791670955126;   // 2 / sqrt(pi)
    const double rinv = rsqrt(r2);
    const double inv_r2 = rinv * rinv;
    const double inv_r3 = inv_r2 * rinv;
    const double r = r2 * rinv;
    if (r2 < small2) {
        const double x = alpha * r;
        const double s2 = r2 + eps2;
        const double si = rsqrt(s2);
        return (-erf(x) + sp * x * exp(-x * x)) * inv_r3 + si * si * si;
    }
    const double u = eps2 * inv_r2;
    double soft;
    if (u < 1e-3) {
        // (1 + u)^{-3/2} - 1 = -3/2 u + 15/8 u^2 - 35/16 u^3 + 315/128 u^4 - ...
        soft = u * (-1.5 + u * (1.875 + u * (-2.1875 + u * 2.4609375)));
    } else {
        const double t = r * rsqrt(r2 + eps2);   // r / sqrt(r^2 + eps2)
        soft = t * t * t - 1.0;
    }
    double f = soft * inv_r3;
    if (r2 < rc2) f += g_of(alpha * r) * inv_r3;
    return f;
}

// Sources in Morton order of their 128^3 cell: 32 consecutive sorted
// sources lie close together, so the lanes of a warp (one target, a source
// each) take the same branches of the pair factor but where the target's
// distance to that small group straddles r_cut.
__device__ __forceinline__ unsigned long long spread3(unsigned v) {
    unsigned long long x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__global__ void k_src_keys(const Pm3Parts s, double inv_box, unsigned long long* __restrict__ keys,
                           unsigned* __restrict__ vals) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.n) return;
    unsigned c[3];
    for (int d = 0; d < 3; ++d) {
        const double f = s.x[d][j] * inv_box * (1 << MORTON_BITS);
        const int ci = f >= 0.0 ? (int)f : 0;               // NaN and negatives go to cell 0
        c[d] = (unsigned)min(ci, (1 << MORTON_BITS) - 1);
    }
    keys[j] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
    vals[j] = (unsigned)j;
}

__global__ void k_src_gather(const Pm3Parts s, const unsigned* __restrict__ order, double4* __restrict__ sorted,
                             int* __restrict__ rank) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    const unsigned j = order[p];
    sorted[p] = make_double4(s.x[0][j], s.x[1][j], s.x[2][j], s.m ? s.m[j] : s.mass_const);
    rank[j] = (int)p;
}

// Real-space sum: a warp per target, lane l taking sources j0 + l, j0 + l +
// 32, ... of the sorted list (coalesced loads; the block's warps read the
// same stretches, so most come from L1); the lanes' sums are added by
// shuffles at the end. The source list is split into chunks (grid.y) for
// parallelism; partials per chunk.
__global__ void __launch_bounds__(RS_NT) k_ewald_real(const double4* __restrict__ src, long long n_src,
                                                      const int* __restrict__ rank, const Targets T, double G,
                                                      double box, double alpha, double rc2, double eps2,
                                                      double small2, long long per_chunk, double* __restrict__ part) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long i = (long long)blockIdx.x * RS_WARPS + warp;
    if (i >= T.n) return;
    const double xi = T.t[0][i], yi = T.t[1][i], zi = T.t[2][i];
    const long long self = T.self && T.self[i] >= 0 && T.self[i] < n_src ? rank[T.self[i]] : -1;
    const double inv_box = 1.0 / box;
    const long long j0 = (long long)blockIdx.y * per_chunk;
    const long long j1 = min(n_src, j0 + per_chunk);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (long long j = j0 + lane; j < j1; j += 32) {
        const double4 sj = src[j];
        double dx = xi - sj.x, dy = yi - sj.y, dz = zi - sj.z;
        dx -= box * rint(dx * inv_box);
        dy -= box * rint(dy * inv_box);
        dz -= box * rint(dz * inv_box);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > 0.0 && j != self && (eps2 > 0.0 || r2 < rc2)) {
            const double f = G * sj.w * ewald_pair(r2, alpha, eps2, rc2, small2);
            ax -= f * dx;
            ay -= f * dy;
            az -= f * dz;
        }
    }
    for (int o = 16; o; o >>= 1) {
        ax += __shfl_down_sync(0xffffffffu, ax, o);
        ay += __shfl_down_sync(0xffffffffu, ay, o);
        az += __shfl_down_sync(0xffffffffu, az, o);
    }
    if (lane == 0) {
        part[((long long)blockIdx.y * 3 + 0) * T.n + i] = ax;
        part[((long long)blockIdx.y * 3 + 1) * T.n + i] = ay;
        part[((long long)blockIdx.y * 3 + 2) * T.n + i] = az;
    }
}

__global__ void k_ewald_final(const Targets T, const double* __restrict__ part, int chunks, double G, double box,
                              const int* __restrict__ hvec, const double* __restrict__ coef,
                              const double* __restrict__ sc, int nk, double* ox, double* oy, double* oz) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.n) return;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int c = 0; c < chunks; ++c) {
        ax += part[((long long)c * 3 + 0) * T.n + i];
        ay += part[((long long)c * 3 + 1) * T.n + i];
        az += part[((long long)c * 3 + 2) * T.n + i];
    }
    const double xi = T.t[0][i] / box, yi = T.t[1][i] / box, zi = T.t[2][i] / box;
    const double kscale = 2.0 * PI / box;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    for (int k = 0; k < nk; ++k) {
        const int hx = hvec[3 * k], hy = hvec[3 * k + 1], hz = hvec[3 * k + 2];
        double sn, cs;
        sincospi(2.0 * (hx * xi + hy * yi + hz * zi), &sn, &cs);
        const double f = coef[k] * (sn * sc[2 * k] - cs * sc[2 * k + 1]);
        rx += f * hx;
        ry += f * hy;
        rz += f * hz;
    }
    ox[i] = ax - G * kscale * rx;
    oy[i] = ay - G * kscale * ry;
    oz[i] = az - G * kscale * rz;
}

int check_src(sss_ctx* ctx, const sss_pm3_particles* s) {
    if (!s || s->n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "bad source state");
    if (s->n > 0 && (!s->x[0] || !s->x[1] || !s->x[2])) return sss_set_err(ctx, SSS_ERR_ARG, "NULL source array");
    return SSS_OK;
}

}  // namespace

extern "C" int sss_ewald_structure(sss_ctx* ctx, const sss_pm3_particles* src, double box, const int* hvec, int nk,
                                   int hmax, double* sc, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    int rc = check_src(ctx, src);
    if (rc) return rc;
    if (nk < 0 || (nk > 0 && (!hvec || !sc))) return sss_set_err(ctx, SSS_ERR_ARG, "bad k-vector list");
    if (!(box > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "box must be > 0");
    if (hmax < 1 || hmax > 40) return sss_set_err(ctx, SSS_ERR_ARG, "hmax must be in [1, 40]");
    if (nk == 0) return SSS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int kb = (nk + SK_NT - 1) / SK_NT;
    int chunks = std::max(1, (ctx->num_sms * 4 + kb - 1) / kb);
    if (src->n == 0) chunks = 1;
    const long long per_chunk = std::max<long long>(1, (src->n + chunks - 1) / chunks);
    chunks = (int)std::max<long long>(1, (src->n + per_chunk - 1) / per_chunk);
    void* scr = nullptr;
    rc = sss_scratch(ctx, (size_t)chunks * nk * sizeof(double2), &scr);
    if (rc) return rc;
    const size_t smem = (size_t)SK_TILE * 3 * (hmax + 1) * sizeof(double2);
    SSS_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ewald_sk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_ewald_sk<<<dim3(kb, chunks), SK_NT, smem, st>>>(pm3_parts(src), 1.0 / box, hvec, nk, hmax, per_chunk,
                                                     (double2*)scr);
    SSS_LAUNCH_CHECK(ctx, "k_ewald_sk");
    k_ewald_sk_reduce<<<(nk + 255) / 256, 256, 0, st>>>((const double2*)scr, nk, chunks, sc);
    SSS_LAUNCH_CHECK(ctx, "k_ewald_sk_reduce");
    return SSS_OK;
}

extern "C" int sss_ewald_accel(sss_ctx* ctx, const sss_pm3_particles* src, const double* const* t,
                               const int64_t* self_idx, int64_t n_tgt, double G, double box, double alpha,
                               double r_cut, double eps2, const int* hvec, const double* coef, const double* sc,
                               int nk, double* const* out, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    int rc = check_src(ctx, src);
    if (rc) return rc;
    if (n_tgt < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative target count");
    if (n_tgt == 0) return SSS_OK;
    if (!t || !t[0] || !t[1] || !t[2] || !out || !out[0] || !out[1] || !out[2])
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL target or output array");
    if (!(box > 0.0) || !(alpha > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "box and alpha must be > 0");
    if (!(r_cut > 0.0) || r_cut > 0.5 * box) return sss_set_err(ctx, SSS_ERR_ARG, "r_cut must be in (0, box/2]");
    if (!(alpha * r_cut <= G_XMAX)) return sss_set_err(ctx, SSS_ERR_ARG, "alpha * r_cut must be <= %g", G_XMAX);
    if (nk < 0 || (nk > 0 && (!hvec || !coef || !sc))) return sss_set_err(ctx, SSS_ERR_ARG, "bad k-vector list");
    cudaStream_t st = (cudaStream_t)stream;
    rc = ensure_gtab(ctx, st);
    if (rc) return rc;
    Targets T;
    for (int c = 0; c < 3; ++c) T.t[c] = t[c];
    T.self = (const long long*)self_idx;
    T.n = n_tgt;
    const long long n = src->n;
    if (n >= (1LL << 31)) return sss_set_err(ctx, SSS_ERR_ARG, "at most 2^31 - 1 sources");
    const int tb = (int)((n_tgt + RS_WARPS - 1) / RS_WARPS);
    int chunks = std::max(1, (ctx->num_sms * 8 + tb - 1) / tb);
    const long long per_chunk = std::max<long long>(1024, (n + chunks - 1) / chunks);
    chunks = (int)std::max<long long>(1, (n + per_chunk - 1) / per_chunk);
    // scratch: partials | sorted sources | rank | keys, values (x2) | sort scratch
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_part = take((size_t)chunks * 3 * n_tgt * sizeof(double));
    const size_t o_sorted = take((size_t)n * sizeof(double4));
    const size_t o_rank = take((size_t)n * sizeof(int));
    const size_t o_k0 = take((size_t)n * 8), o_k1 = take((size_t)n * 8);
    const size_t o_v0 = take((size_t)n * 4), o_v1 = take((size_t)n * 4);
    const size_t o_rs = take(sss_dev::radix_scratch(n) * 8);
    void* scr = nullptr;
    rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* base = (char*)scr;
    double* part = (double*)(base + o_part);
    double4* sorted = (double4*)(base + o_sorted);
    int* rank = (int*)(base + o_rank);
    unsigned long long* k0 = (unsigned long long*)(base + o_k0);
    unsigned long long* k1 = (unsigned long long*)(base + o_k1);
    unsigned* v0 = (unsigned*)(base + o_v0);
    unsigned* v1 = (unsigned*)(base + o_v1);
    const Pm3Parts ps = pm3_parts(src);
    if (n > 0) {
        const unsigned nb = (unsigned)((n + 255) / 256);
        k_src_keys<<<nb, 256, 0, st>>>(ps, 1.0 / box, k0, v0);
        SSS_LAUNCH_CHECK(ctx, "k_src_keys");
        SSS_CUDA_TRY(ctx, sss_dev::radix_sort(k0, v0, k1, v1, n, (long long*)(base + o_rs), st, ctx->d_status));
        k_src_gather<<<nb, 256, 0, st>>>(ps, v0, sorted, rank);
        SSS_LAUNCH_CHECK(ctx, "k_src_gather");
    }
    const double small2 = std::max(1000.0 * eps2, (0.5 / alpha) * (0.5 / alpha));
    k_ewald_real<<<dim3(tb, chunks), RS_NT, 0, st>>>(sorted, n, rank, T, G, box, alpha, r_cut * r_cut, eps2, small2,
                                                    per_chunk, part);
    SSS_LAUNCH_CHECK(ctx, "k_ewald_real");
    k_ewald_final<<<(unsigned)((n_tgt + 127) / 128), 128, 0, st>>>(T, part, chunks, G, box, hvec, coef,
                                                                   sc, nk, out[0], out[1], out[2]);
    SSS_LAUNCH_CHECK(ctx, "k_ewald_final");
    return SSS_OK;
}

extern "C" int sss_ewald_gtab(double* out, int64_t cap, int* n_int, double* h) {
    if (!out || !n_int || !h || cap < (int64_t)G_NI * (G_DEG + 1)) return SSS_ERR_ARG;
    build_gtab(out);
    *n_int = G_NI;
    *h = G_H;
    return SSS_OK;
}
