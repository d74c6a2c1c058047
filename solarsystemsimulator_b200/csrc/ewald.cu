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
// products); k_ewald_real is the target x source real-space sum (sources
// staged through shared memory, the source list split into chunks for
// parallelism; partials added in chunk order); k_ewald_final adds the
// partials and the reciprocal part per target. Deterministic.

#include "pm3d.cuh"

#include <algorithm>

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr int SK_NT = 256;      // k vectors per CTA
constexpr int SK_TILE = 32;     // particles per staged table
constexpr int RS_NT = 128;      // targets per CTA of the real-space sum

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

// the factor f(r) of one pair, a = -G m f d (see the file comment). The
// powers of r come from one reciprocal square root (CUDA's double rsqrt,
// 1 ulp) instead of a square root and two divisions.
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
    if (r2 < rc2) {
        const double x = alpha * r;
        f += (erfc(x) + sp * x * exp(-x * x)) * inv_r3;
    }
    return f;
}

__global__ void __launch_bounds__(RS_NT) k_ewald_real(const Pm3Parts s, const Targets T, double G, double box,
                                                      double alpha, double rc2, double eps2, double small2,
                                                      long long per_chunk, double* __restrict__ part) {
    __shared__ double4 src[RS_NT];
    const long long i = (long long)blockIdx.x * RS_NT + threadIdx.x;
    const bool ok = i < T.n;
    double xi = 0.0, yi = 0.0, zi = 0.0;
    long long self = -1;
    if (ok) {
        xi = T.t[0][i];
        yi = T.t[1][i];
        zi = T.t[2][i];
        self = T.self ? T.self[i] : -1;
    }
    const double inv_box = 1.0 / box;
    const long long j0 = (long long)blockIdx.y * per_chunk;
    const long long j1 = min(s.n, j0 + per_chunk);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (long long b = j0; b < j1; b += RS_NT) {
        const int cnt = (int)min((long long)RS_NT, j1 - b);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const long long j = b + threadIdx.x;
            src[threadIdx.x] = make_double4(s.x[0][j], s.x[1][j], s.x[2][j], s.m ? s.m[j] : s.mass_const);
        }
        __syncthreads();
        for (int q = 0; q < cnt; ++q) {
            const double4 sj = src[q];
            double dx = xi - sj.x, dy = yi - sj.y, dz = zi - sj.z;
            dx -= box * rint(dx * inv_box);
            dy -= box * rint(dy * inv_box);
            dz -= box * rint(dz * inv_box);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 0.0 && b + q != self && (eps2 > 0.0 || r2 < rc2)) {
                const double f = G * sj.w * ewald_pair(r2, alpha, eps2, rc2, small2);
                ax -= f * dx;
                ay -= f * dy;
                az -= f * dz;
            }
        }
    }
    if (ok) {
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
    if (nk < 0 || (nk > 0 && (!hvec || !coef || !sc))) return sss_set_err(ctx, SSS_ERR_ARG, "bad k-vector list");
    cudaStream_t st = (cudaStream_t)stream;
    Targets T;
    for (int c = 0; c < 3; ++c) T.t[c] = t[c];
    T.self = (const long long*)self_idx;
    T.n = n_tgt;
    const int tb = (int)((n_tgt + RS_NT - 1) / RS_NT);
    int chunks = std::max(1, (ctx->num_sms * 8 + tb - 1) / tb);
    const long long per_chunk = std::max<long long>(RS_NT, (src->n + chunks - 1) / chunks);
    chunks = (int)std::max<long long>(1, (src->n + per_chunk - 1) / per_chunk);
    void* scr = nullptr;
    rc = sss_scratch(ctx, (size_t)chunks * 3 * n_tgt * sizeof(double), &scr);
    if (rc) return rc;
    const double small2 = std::max(1000.0 * eps2, (0.5 / alpha) * (0.5 / alpha));
    k_ewald_real<<<dim3(tb, chunks), RS_NT, 0, st>>>(pm3_parts(src), T, G, box, alpha, r_cut * r_cut, eps2,
                                                    small2, per_chunk, (double*)scr);
    SSS_LAUNCH_CHECK(ctx, "k_ewald_real");
    k_ewald_final<<<(unsigned)((n_tgt + 127) / 128), 128, 0, st>>>(T, (const double*)scr, chunks, G, box, hvec, coef,
                                                                   sc, nk, out[0], out[1], out[2]);
    SSS_LAUNCH_CHECK(ctx, "k_ewald_final");
    return SSS_OK;
}
