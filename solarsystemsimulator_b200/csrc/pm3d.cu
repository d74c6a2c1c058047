// 3-D periodic particle mesh for sm_100a: the reference's PM cycle
// (TODO.md:225-253: deposit, Poisson solve in Fourier space, interpolation
// with the deposit's stencil; 2-D code pm_kernel.py:63-154) on an n^3 f32
// mesh in a periodic box.
//
//   deposit  : CIC, positions f64, weights f32, warp-aggregated atomics:
//              lanes of a warp whose particles share a cell add their
//              weights in registers first and one lane issues the atomics.
//   solve    : cuFFT R2C -> k_spectrum3 (Green's function -4 pi G / k^2,
//              divided by the CIC window W(k)^deconv (2: deposit and
//              gather) and filtered by exp(-k^2 r_split^2), the spectral
//              gradient a_d = -i k_d phi, the 1/n^3 of the inverse
//              transform; one read of rho_k, three writes) -> one batched
//              C2R for the three components. cuFFT performs the transforms
//              only.
//   gather   : trilinear (CIC) interpolation of the three f32 meshes into
//              f64 accelerations, fused with the KDK epilogue.
//
// HBM per step at 1,048,576 particles on 256^3: deposit reads 24 B per
// particle and makes 8 atomic f32 updates, the spectrum kernel moves
// 32 B per mode, the gather reads 24 B per particle plus 24 f32 mesh values
// (L2-resident for a 64 MiB mesh) and writes the state.

#include "pm3d.cuh"

#include <algorithm>

namespace {

unsigned blocks_for(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

int cufft_err(sss_ctx* ctx, cufftResult r, const char* what) {
    return sss_set_err(ctx, SSS_ERR_CUDA, "%s: cuFFT error %d", what, (int)r);
}

constexpr unsigned FULL = 0xffffffffu;

// Sum of v over the lanes in `peers` (this lane's group, lane order); all 32
// lanes must call it with their own group and the warp's largest group
// size `most`.
__device__ __forceinline__ float group_sum(unsigned peers, unsigned most, float v) {
    const int lane = threadIdx.x & 31;
    float sum = 0.0f;
    unsigned rest = peers;
    for (unsigned k = 0; k < most; ++k) {
        const int src = rest ? __ffs(rest) - 1 : lane;
        const float o = __shfl_sync(FULL, v, src);
        if (rest) {
            sum += o;
            rest &= rest - 1;
        }
    }
    return sum;
}

// Warp-aggregated CIC deposit. Lanes whose particles lie in the same cell
// share all 8 corner nodes: one __match_any_sync on the cell finds them, the
// group's weights are added in registers (lane order) and its lowest lane
// issues one atomic per corner. Particles of different cells that share a
// node still add separately (atomics keep that correct).
__global__ void __launch_bounds__(256) k_deposit3(const Pm3Parts s, int n, double inv_h, double inv_h3,
                                                  float* __restrict__ rho) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (long long base = w0 * 32; base < s.n; base += warps * 32) {
        const long long p = base + lane;
        const bool ok = p < s.n;
        int i[3] = {0, 0, 0};
        double t[3] = {0.0, 0.0, 0.0};
        double mass = 0.0;
        if (ok) {
            for (int c = 0; c < 3; ++c) pm3_cell(s.x[c][p], inv_h, n, i[c], t[c]);
            mass = (s.m ? s.m[p] : s.mass_const) * inv_h3;
        }
        const int cell = ok ? (i[0] * n + i[1]) * n + i[2] : -1;
        const unsigned peers = __match_any_sync(FULL, cell);
        const bool leader = ok && (__ffs(peers) - 1) == lane;
        const unsigned most = __reduce_max_sync(FULL, (unsigned)__popc(peers));
        const int j[3] = {i[0] + 1 == n ? 0 : i[0] + 1, i[1] + 1 == n ? 0 : i[1] + 1, i[2] + 1 == n ? 0 : i[2] + 1};
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int dx = c >> 2, dy = (c >> 1) & 1, dz = c & 1;
            const double w = (dx ? t[0] : 1.0 - t[0]) * (dy ? t[1] : 1.0 - t[1]) * (dz ? t[2] : 1.0 - t[2]);
            float v = (float)(mass * w);
            if (most > 1) v = group_sum(peers, most, v);
            if (leader) {
                const int key = ((dx ? j[0] : i[0]) * n + (dy ? j[1] : i[1])) * n + (dz ? j[2] : i[2]);
                atomicAdd(rho + key, v);
            }
        }
    }
}

// Per-axis tables of the spectrum kernel, index i of a full axis (frequency
// f = i for i < n/2, i - n otherwise): kd = k_i (0 on the Nyquist index:
// the derivative of that mode is dropped so the spectra stay Hermitian),
// k2 = k_i^2, fac = sinc(pi f / n)^(-2 deconv) * exp(-k_i^2 rs2). The
// Green's function factorises: W(k)^-deconv e^{-k^2 rs2} = fac_x fac_y fac_z.
// The half axis of the real transform (iz <= n/2) reads the same tables.
__global__ void k_spectrum_tables(int n, double box, int deconv, double rs2, double* __restrict__ tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int f = i < n / 2 ? i : i - n;
    const double k = 2.0 * 3.14159265358979323846 / box * f;
    double fac = 1.0;
    if (f != 0) {
        const double a = (double)f / (double)n;
        const double sinc = sinpi(a) / (3.14159265358979323846 * a);
        const double s2 = sinc * sinc;
        for (int q = 0; q < deconv; ++q) fac /= s2;
    }
    if (rs2 > 0.0) fac *= exp(-k * k * rs2);
    tab[i] = (i == n / 2) ? 0.0 : k;
    tab[n + i] = k * k;
    tab[2 * n + i] = fac;
}

// Acceleration spectra from the density spectrum (half-complex layout,
// index (ix, iy, iz), iz in [0, n/2]); grid (z blocks, n, n):
// a_d = -i k_d phi, phi = -4 pi G rho_k fac / k^2  ->  a_d = i k_d c rho_k
// with c = 4 pi G fac / (k^2 n^3) (the inverse transform's 1/n^3 folded in).
__global__ void __launch_bounds__(128) k_spectrum3(const float2* __restrict__ rk, int n, double cscale,
                                                   const double* __restrict__ tab, float2* __restrict__ ak) {
    const int nh = n / 2 + 1;
    const int iz = blockIdx.x * blockDim.x + threadIdx.x;
    if (iz >= nh) return;
    const int iy = blockIdx.y, ix = blockIdx.z;
    const long long m = (long long)n * n * nh;
    const long long t = ((long long)ix * n + iy) * nh + iz;
    float2 out[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    if (ix != 0 || iy != 0 || iz != 0) {
        const double* kd = tab;
        const double* k2t = tab + n;
        const double* fac = tab + 2 * n;
        const double k2 = k2t[ix] + k2t[iy] + k2t[iz];
        const double c = cscale * (fac[ix] * fac[iy] * fac[iz]) / k2;
        const float2 r = rk[t];
        const double kk[3] = {kd[ix], kd[iy], kd[iz]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double f = kk[d] * c;
            out[d] = make_float2((float)(-f * (double)r.y), (float)(f * (double)r.x));
        }
    }
    ak[t] = out[0];
    ak[m + t] = out[1];
    ak[2 * m + t] = out[2];
}

__global__ void __launch_bounds__(256) k_gather3(const Pm3Parts s, int n, double inv_h,
                                                 const float* __restrict__ acc, const Pm3Epi e) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    int i[3];
    double t[3];
    for (int c = 0; c < 3; ++c) pm3_cell(s.x[c][p], inv_h, n, i[c], t[c]);
    const int j[3] = {i[0] + 1 == n ? 0 : i[0] + 1, i[1] + 1 == n ? 0 : i[1] + 1, i[2] + 1 == n ? 0 : i[2] + 1};
    const long long n3 = (long long)n * n * n;
    double a[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int dx = c >> 2, dy = (c >> 1) & 1, dz = c & 1;
        const double w = (dx ? t[0] : 1.0 - t[0]) * (dy ? t[1] : 1.0 - t[1]) * (dz ? t[2] : 1.0 - t[2]);
        const long long q = ((long long)(dx ? j[0] : i[0]) * n + (dy ? j[1] : i[1])) * n + (dz ? j[2] : i[2]);
        a[0] += w * (double)__ldg(acc + q);
        a[1] += w * (double)__ldg(acc + n3 + q);
        a[2] += w * (double)__ldg(acc + 2 * n3 + q);
    }
    pm3_epilogue(s, e, p, a[0], a[1], a[2]);
}

__global__ void __launch_bounds__(256) k_kick_drift3(const Pm3Parts s, double hdt, double dt, double box) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    for (int c = 0; c < 3; ++c) {
        const double v = s.v[c][p] + s.a[c][p] * hdt;
        s.v[c][p] = v;
        s.x[c][p] = pm3_wrap(s.x[c][p] + v * dt, box);
    }
}

void pm3_free(sss_pm3* p) {
    if (p->fwd) cufftDestroy(p->fwd);
    if (p->inv3) cufftDestroy(p->inv3);
    cudaFree(p->rho);
    cudaFree(p->lrho);
    cudaFree(p->rk);
    cudaFree(p->ak);
    cudaFree(p->acc);
    cudaFree(p->tab);
    free(p);
}

int check_parts(sss_ctx* ctx, const sss_pm3_particles* s) {
    if (!s) return sss_set_err(ctx, SSS_ERR_ARG, "NULL particle state");
    if (s->n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative particle count");
    if (s->n == 0) return SSS_OK;
    for (int c = 0; c < 3; ++c)
        if (!s->x[c] || !s->v[c] || !s->a[c]) return sss_set_err(ctx, SSS_ERR_ARG, "NULL particle array");
    return SSS_OK;
}

}  // namespace

extern "C" int sss_pm3_create(sss_ctx* ctx, int mesh_n, double box, sss_pm3** out) {
    if (!ctx || !out) return SSS_ERR_ARG;
    *out = nullptr;
    if (mesh_n < 8 || mesh_n > 1024 || (mesh_n & 1))
        return sss_set_err(ctx, SSS_ERR_ARG, "mesh_n must be even and in [8, 1024]");
    if (!(box > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "box must be > 0");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    sss_pm3* p = (sss_pm3*)calloc(1, sizeof(sss_pm3));
    p->ctx = ctx;
    p->n = mesh_n;
    p->box = box;
    const size_t n3 = (size_t)mesh_n * mesh_n * mesh_n;
    const size_t m = (size_t)mesh_n * mesh_n * (mesh_n / 2 + 1);
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&p->rho, n3 * sizeof(float));
    e = e ? e : cudaMalloc(&p->lrho, n3 * sizeof(float));
    e = e ? e : cudaMalloc(&p->rk, m * sizeof(float2));
    e = e ? e : cudaMalloc(&p->ak, 3 * m * sizeof(float2));
    e = e ? e : cudaMalloc(&p->acc, 3 * n3 * sizeof(float));
    e = e ? e : cudaMalloc(&p->tab, 3 * (size_t)mesh_n * sizeof(double));
    p->tab_deconv = -1;
    if (e != cudaSuccess) {
        pm3_free(p);
        return sss_cuda_err(ctx, e, "cudaMalloc (pm3)");
    }
    cufftResult r = cufftPlan3d(&p->fwd, mesh_n, mesh_n, mesh_n, CUFFT_R2C);
    if (r == CUFFT_SUCCESS) {
        int dims[3] = {mesh_n, mesh_n, mesh_n};
        r = cufftPlanMany(&p->inv3, 3, dims, nullptr, 1, (int)m, nullptr, 1, (int)n3, CUFFT_C2R, 3);
    }
    if (r != CUFFT_SUCCESS) {
        pm3_free(p);
        return cufft_err(ctx, r, "cufftPlan (pm3)");
    }
    *out = p;
    return SSS_OK;
}

extern "C" void sss_pm3_destroy(sss_pm3* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaDeviceSynchronize();
    pm3_free(p);
}

extern "C" int sss_pm3_meshes(sss_pm3* p, float** rho, float** accel) {
    if (!p) return SSS_ERR_ARG;
    if (rho) *rho = p->rho;
    if (accel) *accel = p->acc;
    return SSS_OK;
}

extern "C" int sss_pm3_density(sss_pm3* p, const sss_pm3_particles* s, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    int rc = check_parts(ctx, s);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const long long n3 = (long long)p->n * p->n * p->n;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(p->rho, 0, (size_t)n3 * sizeof(float), st));
    if (s->n == 0) return SSS_OK;
    const double inv_h = p->n / p->box;
    const double h = p->box / p->n;
    const int blocks = (int)std::min<long long>((s->n + 255) / 256, (long long)ctx->num_sms * 8);
    k_deposit3<<<blocks, 256, 0, st>>>(pm3_parts(s), p->n, inv_h, 1.0 / (h * h * h), p->rho);
    SSS_LAUNCH_CHECK(ctx, "k_deposit3");
    return SSS_OK;
}

extern "C" int sss_pm3_solve(sss_pm3* p, double G, int deconv, double r_split, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    if (deconv < 0 || deconv > 4) return sss_set_err(ctx, SSS_ERR_ARG, "deconv must be in [0, 4]");
    if (!(r_split >= 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "r_split must be >= 0");
    cudaStream_t st = (cudaStream_t)stream;
    cufftSetStream(p->fwd, st);
    cufftSetStream(p->inv3, st);
    cufftResult r = cufftExecR2C(p->fwd, p->rho, (cufftComplex*)p->rk);
    if (r != CUFFT_SUCCESS) return cufft_err(ctx, r, "cufftExecR2C");
    const double rs2 = r_split * r_split;
    if (p->tab_deconv != deconv || p->tab_rs2 != rs2) {
        k_spectrum_tables<<<blocks_for(p->n, 128), 128, 0, st>>>(p->n, p->box, deconv, rs2, p->tab);
        SSS_LAUNCH_CHECK(ctx, "k_spectrum_tables");
        p->tab_deconv = deconv;
        p->tab_rs2 = rs2;
    }
    const int nh = p->n / 2 + 1;
    const double cscale = 4.0 * 3.14159265358979323846 * G / ((double)p->n * p->n * p->n);
    k_spectrum3<<<dim3((nh + 127) / 128, p->n, p->n), 128, 0, st>>>(p->rk, p->n, cscale, p->tab, p->ak);
    SSS_LAUNCH_CHECK(ctx, "k_spectrum3");
    r = cufftExecC2R(p->inv3, (cufftComplex*)p->ak, p->acc);
    if (r != CUFFT_SUCCESS) return cufft_err(ctx, r, "cufftExecC2R");
    return SSS_OK;
}

extern "C" int sss_pm3_gather(sss_pm3* p, const sss_pm3_particles* s, int mode, double hdt, double dt,
                              float* snap, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    int rc = check_parts(ctx, s);
    if (rc) return rc;
    if (mode < SSS_PM3_FORCE || mode > SSS_PM3_KICK_DRIFT) return sss_set_err(ctx, SSS_ERR_ARG, "bad mode");
    if (s->n == 0) return SSS_OK;
    Pm3Epi e{mode, hdt, dt, p->box, snap};
    k_gather3<<<blocks_for(s->n, 256), 256, 0, (cudaStream_t)stream>>>(pm3_parts(s), p->n, p->n / p->box, p->acc,
                                                                      e);
    SSS_LAUNCH_CHECK(ctx, "k_gather3");
    return SSS_OK;
}

extern "C" int sss_pm3_kick_drift(sss_pm3* p, const sss_pm3_particles* s, double hdt, double dt, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    int rc = check_parts(ctx, s);
    if (rc) return rc;
    if (s->n == 0) return SSS_OK;
    k_kick_drift3<<<blocks_for(s->n, 256), 256, 0, (cudaStream_t)stream>>>(pm3_parts(s), hdt, dt, p->box);
    SSS_LAUNCH_CHECK(ctx, "k_kick_drift3");
    return SSS_OK;
}
