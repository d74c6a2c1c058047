// Particle-mesh forces for sm_100a: replaces the 2-D isolated PM of the
// reference (backend/pm_kernel.py:34-293). cuFFT performs only the
// transforms; deposit, kernel build, spectrum multiply, gather and the KDK
// integration are kernels of this file.
//
// 2-D isolated (Hockney-James): masses are deposited by cloud-in-cell
// straight into the zero-padded 2N x 2N grid, transformed (D2Z), multiplied
// by the transforms of the softened force kernels K_x, K_y (with the inverse
// transform's 1/(2N)^2 folded in), transformed back (2x Z2D) and read back
// bilinearly with the deposit's stencil. f64 throughout, as the reference.

#include "sss_internal.cuh"

#include <cufft.h>

namespace {

// ------------------------------------------------------------ 2-D kernels

// K(d) = -G d / (|d|^2 + eps2)^(3/2) on the padded grid, offsets wrapped so
// that index m maps to m (m < N) or m - 2N (pm_kernel.py:42-59).
__global__ void k_force_kernels_2d(int n, double h, double eps2, double G, double* __restrict__ kx,
                                   double* __restrict__ ky) {
    const int np = 2 * n;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)np * np) return;
    const int i = (int)(t / np), j = (int)(t % np);
    const double oi = (double)(i < n ? i : i - np), oj = (double)(j < n ? j : j - np);
    const double dx = __dmul_rn(oi, h), dy = __dmul_rn(oj, h);
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), eps2);
    const double inv_r3 = __ddiv_rn(1.0, __dmul_rn(r2, sqrt(r2)));
    kx[t] = __dmul_rn(__dmul_rn(-G, dx), inv_r3);
    ky[t] = __dmul_rn(__dmul_rn(-G, dy), inv_r3);
}

// CIC corner index/weights of the reference (pm_kernel.py:63-90): cell
// clipped to [0, N-2], fractional offsets from the clipped cell.
__device__ __forceinline__ void cic2(double gx, double gy, double x0, double y0, double h, int n, int& i,
                                     int& j, double& tx, double& ty) {
    const double fx = __ddiv_rn(__dsub_rn(gx, x0), h);
    const double fy = __ddiv_rn(__dsub_rn(gy, y0), h);
    i = (int)floor(fx);
    j = (int)floor(fy);
    i = min(max(i, 0), n - 2);
    j = min(max(j, 0), n - 2);
    tx = __dsub_rn(fx, (double)i);
    ty = __dsub_rn(fy, (double)j);
}

// deposit into the padded (2N x 2N, row stride 2N) array
__global__ void k_cic_deposit_2d(const double* __restrict__ gx, const double* __restrict__ gy,
                                 const double* __restrict__ gm, long long np_, int n, double x0, double y0,
                                 double h, double* __restrict__ rho_pad) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np_) return;
    int i, j;
    double tx, ty;
    cic2(gx[p], gy[p], x0, y0, h, n, i, j, tx, ty);
    const double m = gm[p];
    const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
    const long long s = 2LL * n;
    atomicAdd(&rho_pad[(long long)i * s + j], __dmul_rn(__dmul_rn(m, ux), uy));
    atomicAdd(&rho_pad[(long long)(i + 1) * s + j], __dmul_rn(__dmul_rn(m, tx), uy));
    atomicAdd(&rho_pad[(long long)i * s + (j + 1)], __dmul_rn(__dmul_rn(m, ux), ty));
    atomicAdd(&rho_pad[(long long)(i + 1) * s + (j + 1)], __dmul_rn(__dmul_rn(m, tx), ty));
}

// F_x = rho_k * FK_x * scale, F_y = rho_k * FK_y * scale (complex, numpy order)
__global__ void k_spectrum_mul_2d(const double2* __restrict__ fr, const double2* __restrict__ fkx,
                                  const double2* __restrict__ fky, long long m, double scale,
                                  double2* __restrict__ outx, double2* __restrict__ outy) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const double2 a = fr[t], bx = fkx[t], by = fky[t];
    double2 cx, cy;
    cx.x = __dmul_rn(__dsub_rn(__dmul_rn(a.x, bx.x), __dmul_rn(a.y, bx.y)), scale);
    cx.y = __dmul_rn(__dadd_rn(__dmul_rn(a.x, bx.y), __dmul_rn(a.y, bx.x)), scale);
    cy.x = __dmul_rn(__dsub_rn(__dmul_rn(a.x, by.x), __dmul_rn(a.y, by.y)), scale);
    cy.y = __dmul_rn(__dadd_rn(__dmul_rn(a.x, by.y), __dmul_rn(a.y, by.x)), scale);
    outx[t] = cx;
    outy[t] = cy;
}

// bilinear read of the [0:N, 0:N] crop of the 2N x 2N fields (pm_kernel.py:93-107)
__global__ void k_cic_gather_2d(const double* __restrict__ px, const double* __restrict__ py, long long np_,
                                int n, double x0, double y0, double h, const double* __restrict__ fx_pad,
                                const double* __restrict__ fy_pad, double* __restrict__ ax,
                                double* __restrict__ ay) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np_) return;
    int i, j;
    double tx, ty;
    cic2(px[p], py[p], x0, y0, h, n, i, j, tx, ty);
    const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
    const long long s = 2LL * n;
    const long long c00 = (long long)i * s + j, c10 = c00 + s, c01 = c00 + 1, c11 = c10 + 1;
    // f[..] * (1 - tx) * (1 - ty) + ... evaluated left to right, as the reference
    const double* F[2] = {fx_pad, fy_pad};
    double out[2];
    for (int q = 0; q < 2; ++q) {
        const double* f = F[q];
        const double t00 = __dmul_rn(__dmul_rn(f[c00], ux), uy);
        const double t10 = __dmul_rn(__dmul_rn(f[c10], tx), uy);
        const double t01 = __dmul_rn(__dmul_rn(f[c01], ux), ty);
        const double t11 = __dmul_rn(__dmul_rn(f[c11], tx), ty);
        out[q] = __dadd_rn(__dadd_rn(__dadd_rn(t00, t10), t01), t11);
    }
    ax[p] = out[0];
    ay[p] = out[1];
}

// bilinear read of one caller-held N x N field with row stride ld (_cic_gather, pm_kernel.py:93-107)
__global__ void k_cic_gather_field_2d(const double* __restrict__ px, const double* __restrict__ py, long long np_,
                                      int n, long long ld, double x0, double y0, double h,
                                      const double* __restrict__ f, double* __restrict__ out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np_) return;
    int i, j;
    double tx, ty;
    cic2(px[p], py[p], x0, y0, h, n, i, j, tx, ty);
    const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
    const long long c00 = (long long)i * ld + j, c10 = c00 + ld, c01 = c00 + 1, c11 = c10 + 1;
    const double t00 = __dmul_rn(__dmul_rn(f[c00], ux), uy);
    const double t10 = __dmul_rn(__dmul_rn(f[c10], tx), uy);
    const double t01 = __dmul_rn(__dmul_rn(f[c01], ux), ty);
    const double t11 = __dmul_rn(__dmul_rn(f[c11], tx), ty);
    out[p] = __dadd_rn(__dadd_rn(__dadd_rn(t00, t10), t01), t11);
}

// min/max of x and y: out[0..3] = xmin, xmax, ymin, ymax (two-pass: blocks -> final)
__global__ void k_bbox_2d(const double* __restrict__ x, const double* __restrict__ y, long long n,
                          double* __restrict__ part) {
    __shared__ double s[4][8];
    double a = 1e308, b = -1e308, c = 1e308, d = -1e308;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        a = fmin(a, x[i]); b = fmax(b, x[i]);
        c = fmin(c, y[i]); d = fmax(d, y[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        c = fmin(c, __shfl_xor_sync(0xffffffffu, c, o));
        d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { s[0][w] = a; s[1][w] = b; s[2][w] = c; s[3][w] = d; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            a = fmin(a, s[0][k]); b = fmax(b, s[1][k]); c = fmin(c, s[2][k]); d = fmax(d, s[3][k]);
        }
        part[4 * blockIdx.x + 0] = a;
        part[4 * blockIdx.x + 1] = b;
        part[4 * blockIdx.x + 2] = c;
        part[4 * blockIdx.x + 3] = d;
    }
}

__global__ void k_bbox_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 1e308, b = -1e308, c = 1e308, d = -1e308;
    for (int k = 0; k < nb; ++k) {
        a = fmin(a, part[4 * k]); b = fmax(b, part[4 * k + 1]);
        c = fmin(c, part[4 * k + 2]); d = fmax(d, part[4 * k + 3]);
    }
    out[0] = a; out[1] = b; out[2] = c; out[3] = d;
}

// KDK pieces (pm_kernel.py:264-273): v += hdt*a; x += dt*v  /  v += hdt*a
__global__ void k_kick_drift_2d(double* __restrict__ x, double* __restrict__ y, double* __restrict__ vx,
                                double* __restrict__ vy, const double* __restrict__ ax,
                                const double* __restrict__ ay, long long n, double hdt, double dt, int drift) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double nvx = __dadd_rn(vx[i], __dmul_rn(hdt, ax[i]));
    const double nvy = __dadd_rn(vy[i], __dmul_rn(hdt, ay[i]));
    vx[i] = nvx;
    vy[i] = nvy;
    if (drift) {
        x[i] = __dadd_rn(x[i], __dmul_rn(dt, nvx));
        y[i] = __dadd_rn(y[i], __dmul_rn(dt, nvy));
    }
}

__global__ void k_snap_2d(const double* __restrict__ a, long long n, float* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)a[i];
}

unsigned blocks_for(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

int cufft_err(sss_ctx* ctx, cufftResult r, const char* what) {
    return sss_set_err(ctx, SSS_ERR_CUDA, "%s: cuFFT error %d", what, (int)r);
}

}  // namespace

// ------------------------------------------------------------------ C ABI

struct sss_pm2d {
    sss_ctx* ctx;
    int n;                 // grid_n
    cufftHandle fwd, inv;  // D2Z / Z2D on (2N, 2N)
    double* kx;            // real work (2N x 2N) for the kernels / deposit
    double* ky;
    double2* fkx;          // (2N, N+1) spectra of the force kernels
    double2* fky;
    double2* fr;           // spectrum of the density
    double2* sx;           // product spectra
    double2* sy;
    double* fieldx;        // (2N x 2N) real fields
    double* fieldy;
    double* bb_part;       // bbox partials
    double* bb;            // bbox result (4)
};

static int pm2d_free(sss_pm2d* p) {
    if (!p) return SSS_OK;
    if (p->fwd) cufftDestroy(p->fwd);
    if (p->inv) cufftDestroy(p->inv);
    cudaFree(p->kx); cudaFree(p->ky); cudaFree(p->fkx); cudaFree(p->fky); cudaFree(p->fr);
    cudaFree(p->sx); cudaFree(p->sy); cudaFree(p->fieldx); cudaFree(p->fieldy);
    cudaFree(p->bb_part); cudaFree(p->bb);
    free(p);
    return SSS_OK;
}

extern "C" int sss_pm2d_create(sss_ctx* ctx, int grid_n, sss_pm2d** out) {
    if (!ctx || !out) return SSS_ERR_ARG;
    *out = nullptr;
    if (grid_n < 4 || grid_n > 16384) return sss_set_err(ctx, SSS_ERR_ARG, "grid_n must be in [4, 16384]");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    sss_pm2d* p = (sss_pm2d*)calloc(1, sizeof(sss_pm2d));
    p->ctx = ctx;
    p->n = grid_n;
    const long long np = 2LL * grid_n;
    const size_t real_b = (size_t)np * np * sizeof(double);
    const size_t cplx_b = (size_t)np * (grid_n + 1) * sizeof(double2);
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&p->kx, real_b);
    e = e ? e : cudaMalloc(&p->ky, real_b);
    e = e ? e : cudaMalloc(&p->fkx, cplx_b);
    e = e ? e : cudaMalloc(&p->fky, cplx_b);
    e = e ? e : cudaMalloc(&p->fr, cplx_b);
    e = e ? e : cudaMalloc(&p->sx, cplx_b);
    e = e ? e : cudaMalloc(&p->sy, cplx_b);
    e = e ? e : cudaMalloc(&p->fieldx, real_b);
    e = e ? e : cudaMalloc(&p->fieldy, real_b);
    e = e ? e : cudaMalloc(&p->bb_part, 4 * 1024 * sizeof(double));
    e = e ? e : cudaMalloc(&p->bb, 4 * sizeof(double));
    if (e != cudaSuccess) {
        pm2d_free(p);
        return sss_cuda_err(ctx, e, "cudaMalloc (pm2d)");
    }
    cufftResult r = cufftPlan2d(&p->fwd, (int)np, (int)np, CUFFT_D2Z);
    if (r == CUFFT_SUCCESS) r = cufftPlan2d(&p->inv, (int)np, (int)np, CUFFT_Z2D);
    if (r != CUFFT_SUCCESS) {
        pm2d_free(p);
        return cufft_err(ctx, r, "cufftPlan2d");
    }
    *out = p;
    return SSS_OK;
}

extern "C" void sss_pm2d_destroy(sss_pm2d* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaDeviceSynchronize();
    pm2d_free(p);
}

// Bounding box of (x, y) into bbox4 (device, xmin xmax ymin ymax).
extern "C" int sss_pm2d_bbox(sss_pm2d* p, const double* x, const double* y, int64_t n, double* bbox4,
                             void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    if (n < 1 || !x || !y || !bbox4) return sss_set_err(ctx, SSS_ERR_ARG, "bbox: empty or NULL input");
    cudaStream_t s = (cudaStream_t)stream;
    int nb = (int)((n + 255) / 256);
    if (nb > 1024) nb = 1024;
    k_bbox_2d<<<nb, 256, 0, s>>>(x, y, n, p->bb_part);
    k_bbox_final<<<1, 32, 0, s>>>(p->bb_part, nb, bbox4);
    SSS_LAUNCH_CHECK(ctx, "k_bbox");
    return SSS_OK;
}

// FFTs of the softened force kernels for cell size h (pm_kernel.py:34-60);
// kept inside the plan object until the next call.
extern "C" int sss_pm2d_build_kernels(sss_pm2d* p, double h, double eps2, double G, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    if (!(h > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "h must be > 0");
    cudaStream_t s = (cudaStream_t)stream;
    const long long np = 2LL * p->n;
    k_force_kernels_2d<<<blocks_for(np * np, 256), 256, 0, s>>>(p->n, h, eps2, G, p->kx, p->ky);
    SSS_LAUNCH_CHECK(ctx, "k_force_kernels_2d");
    cufftSetStream(p->fwd, s);
    cufftResult r = cufftExecD2Z(p->fwd, p->kx, (cufftDoubleComplex*)p->fkx);
    if (r == CUFFT_SUCCESS) r = cufftExecD2Z(p->fwd, p->ky, (cufftDoubleComplex*)p->fky);
    if (r != CUFFT_SUCCESS) return cufft_err(ctx, r, "cufftExecD2Z (kernels)");
    return SSS_OK;
}

// Field on the grid from the masses (pm_kernel.py:127-147): deposit into the
// padded grid, D2Z, multiply by the kernel spectra, 2x Z2D. The fields stay
// in the plan object (fieldx/fieldy, 2N x 2N, the [0:N, 0:N] crop valid).
extern "C" int sss_pm2d_field(sss_pm2d* p, const double* gx, const double* gy, const double* gm, int64_t n,
                              double x0, double y0, double h, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    if (n < 0 || (n > 0 && (!gx || !gy || !gm))) return sss_set_err(ctx, SSS_ERR_ARG, "field: bad input");
    cudaStream_t s = (cudaStream_t)stream;
    const long long np = 2LL * p->n;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(p->kx, 0, (size_t)np * np * sizeof(double), s));
    if (n > 0) {
        k_cic_deposit_2d<<<blocks_for(n, 256), 256, 0, s>>>(gx, gy, gm, n, p->n, x0, y0, h, p->kx);
        SSS_LAUNCH_CHECK(ctx, "k_cic_deposit_2d");
    }
    cufftSetStream(p->fwd, s);
    cufftSetStream(p->inv, s);
    cufftResult r = cufftExecD2Z(p->fwd, p->kx, (cufftDoubleComplex*)p->fr);
    if (r != CUFFT_SUCCESS) return cufft_err(ctx, r, "cufftExecD2Z (density)");
    const long long m = np * (p->n + 1);
    k_spectrum_mul_2d<<<blocks_for(m, 256), 256, 0, s>>>(p->fr, p->fkx, p->fky, m, 1.0 / (double)(np * np), p->sx,
                                                         p->sy);
    SSS_LAUNCH_CHECK(ctx, "k_spectrum_mul_2d");
    r = cufftExecZ2D(p->inv, (cufftDoubleComplex*)p->sx, p->fieldx);
    if (r == CUFFT_SUCCESS) r = cufftExecZ2D(p->inv, (cufftDoubleComplex*)p->sy, p->fieldy);
    if (r != CUFFT_SUCCESS) return cufft_err(ctx, r, "cufftExecZ2D");
    return SSS_OK;
}

// Accelerations at (px, py) from the last field (pm_kernel.py:150-154).
extern "C" int sss_pm2d_gather(sss_pm2d* p, const double* px, const double* py, int64_t n, double x0, double y0,
                               double h, double* ax, double* ay, void* stream) {
    if (!p) return SSS_ERR_ARG;
    if (n <= 0) return SSS_OK;
    if (!px || !py || !ax || !ay) return sss_set_err(p->ctx, SSS_ERR_ARG, "gather: NULL");
    k_cic_gather_2d<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(px, py, n, p->n, x0, y0, h, p->fieldx,
                                                                         p->fieldy, ax, ay);
    SSS_LAUNCH_CHECK(p->ctx, "k_cic_gather_2d");
    return SSS_OK;
}

// One field read at (px, py) with the deposit's stencil (_cic_gather, pm_kernel.py:93-107).
extern "C" int sss_pm2d_gather_field(sss_ctx* ctx, const double* field, int grid_n, int64_t ld, const double* px,
                                     const double* py, int64_t n, double x0, double y0, double h, double* out,
                                     void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (grid_n < 2 || ld < grid_n || n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "gather_field: bad sizes");
    if (n == 0) return SSS_OK;
    if (!field || !px || !py || !out) return sss_set_err(ctx, SSS_ERR_ARG, "gather_field: NULL");
    k_cic_gather_field_2d<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(px, py, n, grid_n, ld, x0, y0, h,
                                                                               field, out);
    SSS_LAUNCH_CHECK(ctx, "k_cic_gather_field_2d");
    return SSS_OK;
}

// The [0:N, 0:N] crops of the last field into ax, ay (device, N*N each).
extern "C" int sss_pm2d_fields(sss_pm2d* p, double* ax, double* ay, void* stream) {
    if (!p || !ax || !ay) return SSS_ERR_ARG;
    const size_t n = (size_t)p->n;
    cudaStream_t s = (cudaStream_t)stream;
    SSS_CUDA_TRY(p->ctx, cudaMemcpy2DAsync(ax, n * sizeof(double), p->fieldx, 2 * n * sizeof(double),
                                           n * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
    SSS_CUDA_TRY(p->ctx, cudaMemcpy2DAsync(ay, n * sizeof(double), p->fieldy, 2 * n * sizeof(double),
                                           n * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
    return SSS_OK;
}

// Density grid (N x N crop of the padded deposit) into rho (device, N*N).
extern "C" int sss_pm2d_density(sss_pm2d* p, double* rho, void* stream) {
    if (!p || !rho) return SSS_ERR_ARG;
    const size_t n = (size_t)p->n;
    SSS_CUDA_TRY(p->ctx, cudaMemcpy2DAsync(rho, n * sizeof(double), p->kx, 2 * n * sizeof(double),
                                           n * sizeof(double), n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return SSS_OK;
}

// KDK piece: v += hdt a; if drift: x += dt v.
extern "C" int sss_pm2d_kick_drift(sss_pm2d* p, double* x, double* y, double* vx, double* vy, const double* ax,
                                   const double* ay, int64_t n, double hdt, double dt, int drift, void* stream) {
    if (!p) return SSS_ERR_ARG;
    if (n <= 0) return SSS_OK;
    k_kick_drift_2d<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, y, vx, vy, ax, ay, n, hdt, dt, drift);
    SSS_LAUNCH_CHECK(p->ctx, "k_kick_drift_2d");
    return SSS_OK;
}

// f32 copy of an f64 array (snapshot rows).
extern "C" int sss_pm2d_to_f32(sss_pm2d* p, const double* a, int64_t n, float* out, void* stream) {
    if (!p) return SSS_ERR_ARG;
    if (n <= 0) return SSS_OK;
    k_snap_2d<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(a, n, out);
    SSS_LAUNCH_CHECK(p->ctx, "k_snap_2d");
    return SSS_OK;
}
