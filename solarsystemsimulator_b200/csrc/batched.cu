// Many small independent N-body systems (3..64 bodies each), f64 Yoshida-4,
// integrated in persistent kernels: a TEAM of T lanes (T divides 32) owns
// one system at a time, each lane holds B bodies in registers, and the
// team's positions are broadcast to its lanes by width-T warp shuffles, so a
// system never touches shared or global memory between its first and last
// step. Systems are grouped by body count; each group runs with the (T, B)
// mapping an autotuner chose (solarsystemsimulator_b200/batched.py), and
// all groups of a run are launched together (one CUDA graph on the Python
// side).
//
// Force: a_i = sum_{j != i} G m_j (x_j - x_i) / (|x_j - x_i|^2 + eps2)^(3/2)
// (the reference's pair formula, selfgrav_kernel.py:247-255 / nbody_kernel.py
// :166-187, per system). Step: three KDK velocity-Verlet substeps with the
// Yoshida weights (nbody_kernel.py:64-65, 314-401) and a per-system dt.

#include "sss_internal.cuh"

namespace {

struct BatchArgs {
    double* x[3];            // positions, all systems concatenated
    double* v[3];            // velocities
    const double* m;         // masses
    const int64_t* off;      // [n_sys + 1] body offsets of the systems
    const double* G;         // [n_sys]
    const double* dt;        // [n_sys]
    const int* sys_list;     // systems of this group
    int n_list;
    double eps2;
    int steps;
    double w1, w0;
};

template <int D, int T, int B>
__device__ __forceinline__ void team_accel(const double (&px)[B][3], const double (&pm)[B], int n, int lane_t,
                                           unsigned mask, double G, double eps2, double (&acc)[B][3]) {
#pragma unroll
    for (int b = 0; b < B; ++b) acc[b][0] = acc[b][1] = acc[b][2] = 0.0;
    for (int j = 0; j < n; ++j) {
        const int owner = j % T, slot = j / T;
        double sx = 0.0, sy = 0.0, sz = 0.0, sm = 0.0;
#pragma unroll
        for (int b = 0; b < B; ++b) {
            // the slot index is uniform across the team: select, then shuffle
            if (b == slot) { sx = px[b][0]; sy = px[b][1]; sz = px[b][2]; sm = pm[b]; }
        }
        sx = __shfl_sync(mask, sx, owner, T);
        sy = __shfl_sync(mask, sy, owner, T);
        if (D == 3) sz = __shfl_sync(mask, sz, owner, T);
        sm = __shfl_sync(mask, sm, owner, T);
        const double gm = G * sm;
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int i = lane_t + b * T;
            const double dx = sx - px[b][0], dy = sy - px[b][1];
            const double dz = (D == 3) ? sz - px[b][2] : 0.0;
            double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
            const bool self = (i == j) || (i >= n);
            if (self) r2 = 1.0;
            const double inv = rsqrt(r2);
            const double f = self ? 0.0 : ((gm * inv) * inv) * inv;
            acc[b][0] = fma(f, dx, acc[b][0]);
            acc[b][1] = fma(f, dy, acc[b][1]);
            if (D == 3) acc[b][2] = fma(f, dz, acc[b][2]);
        }
    }
}

template <int D, int T, int B>
__global__ void __launch_bounds__(128) k_batched(const BatchArgs a) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int lane_t = lane % T;
    const int team = gtid / T;
    const int n_teams = (gridDim.x * blockDim.x) / T;
    const unsigned mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (lane - lane_t));
    const double wd[3] = {a.w1, a.w0, a.w1};
    for (int q = team; q < a.n_list; q += n_teams) {
        const int s = a.sys_list[q];
        const int64_t o = a.off[s];
        const int n = (int)(a.off[s + 1] - o);
        if (n > T * B) continue;      // the host maps groups to teams that hold them
        const double G = a.G[s], dt = a.dt[s];
        double px[B][3], pv[B][3], pm[B], acc[B][3];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int i = lane_t + b * T;
            const bool ok = i < n;
            for (int c = 0; c < 3; ++c) {
                px[b][c] = (ok && c < D) ? a.x[c][o + i] : 0.0;
                pv[b][c] = (ok && c < D) ? a.v[c][o + i] : 0.0;
            }
            pm[b] = ok ? a.m[o + i] : 0.0;
        }
        team_accel<D, T, B>(px, pm, n, lane_t, mask, G, a.eps2, acc);
        for (int st = 0; st < a.steps; ++st) {
#pragma unroll
            for (int w = 0; w < 3; ++w) {
                const double h = wd[w] * dt;
                const double hh = 0.5 * h;
#pragma unroll
                for (int b = 0; b < B; ++b)
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        pv[b][c] += acc[b][c] * hh;
                        px[b][c] += pv[b][c] * h;
                    }
                team_accel<D, T, B>(px, pm, n, lane_t, mask, G, a.eps2, acc);
#pragma unroll
                for (int b = 0; b < B; ++b)
#pragma unroll
                    for (int c = 0; c < D; ++c) pv[b][c] += acc[b][c] * hh;
            }
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int i = lane_t + b * T;
            if (i < n)
                for (int c = 0; c < D; ++c) {
                    a.x[c][o + i] = px[b][c];
                    a.v[c][o + i] = pv[b][c];
                }
        }
    }
}

template <int D>
void* pick(int T, int B) {
#define SSS_BT(t, b) if (T == t && B == b) return (void*)k_batched<D, t, b>;
    SSS_BT(1, 1) SSS_BT(1, 2) SSS_BT(1, 4) SSS_BT(1, 8)
    SSS_BT(2, 1) SSS_BT(2, 2) SSS_BT(2, 4) SSS_BT(2, 8)
    SSS_BT(4, 1) SSS_BT(4, 2) SSS_BT(4, 4) SSS_BT(4, 8)
    SSS_BT(8, 1) SSS_BT(8, 2) SSS_BT(8, 4) SSS_BT(8, 8)
    SSS_BT(16, 1) SSS_BT(16, 2) SSS_BT(16, 4)
    SSS_BT(32, 1) SSS_BT(32, 2)
#undef SSS_BT
    return nullptr;
}

}  // namespace

extern "C" int sss_batched_launch(sss_ctx* ctx, int dim, double* const* x, double* const* v, const double* m,
                                  const int64_t* off, const double* G, const double* dt, const int* sys_list,
                                  int n_list, int max_n, int team, int per_lane, double eps2, int steps,
                                  int blocks, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (dim != 2 && dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3");
    if (n_list < 0 || steps < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative count");
    if (n_list == 0 || steps == 0) return SSS_OK;
    if (!x || !v || !m || !off || !G || !dt || !sys_list) return sss_set_err(ctx, SSS_ERR_ARG, "NULL argument");
    void* fn = (dim == 3) ? pick<3>(team, per_lane) : pick<2>(team, per_lane);
    if (!fn) return sss_set_err(ctx, SSS_ERR_ARG, "unsupported team mapping T=%d B=%d", team, per_lane);
    if (max_n < 1 || max_n > team * per_lane)
        return sss_set_err(ctx, SSS_ERR_ARG, "a team of %d lanes x %d bodies cannot hold %d bodies", team, per_lane,
                           max_n);
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    BatchArgs a;
    memset(&a, 0, sizeof(a));
    for (int c = 0; c < dim; ++c) { a.x[c] = x[c]; a.v[c] = v[c]; }
    for (int c = dim; c < 3; ++c) { a.x[c] = x[0]; a.v[c] = v[0]; }
    a.m = m;
    a.off = off;
    a.G = G;
    a.dt = dt;
    a.sys_list = sys_list;
    a.n_list = n_list;
    a.eps2 = eps2;
    a.steps = steps;
    a.w1 = 1.0 / (2.0 - cbrt(2.0));
    a.w0 = -cbrt(2.0) / (2.0 - cbrt(2.0));
    if (blocks <= 0) {
        const long long teams = n_list;
        blocks = (int)((teams * team + 127) / 128);
        if (blocks < 1) blocks = 1;
    }
    void* args[] = {&a};
    SSS_CUDA_TRY(ctx, cudaLaunchKernel(fn, dim3(blocks), dim3(128), args, 0, (cudaStream_t)stream));
    return SSS_OK;
}
