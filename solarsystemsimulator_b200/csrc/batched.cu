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
    // unrolled: the shuffles and pair factors of four sources overlap; the
    // accumulation keeps the source order
#pragma unroll 4
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

// Block per system, for the larger groups (NT = 16, 32 or 64 targets):
// thread (t, c) of NT * S takes
// target t and the sources j = c, c + S, c + 2S, ...; positions and masses
// in shared memory, the S partial forces of a target added in chunk order.
// A force evaluation is n / S dependent pair iterations instead of n, with
// S times the warps in flight. Pair formula and KDK as in k_batched.
template <int D, int NT, int S>
__global__ void __launch_bounds__(NT * S) k_batched_blk(const BatchArgs a) {
    __shared__ double4 sp[NT];
    __shared__ double sa[S][3][NT];
    const int t = threadIdx.x % NT, c = threadIdx.x / NT;
    const double wd[3] = {a.w1, a.w0, a.w1};
    for (int q = blockIdx.x; q < a.n_list; q += gridDim.x) {
        const int sys = a.sys_list[q];
        const int64_t o = a.off[sys];
        const int n = (int)(a.off[sys + 1] - o);
        if (n > NT) continue;         // the host maps groups to blocks that hold them
        const double G = a.G[sys], dt = a.dt[sys];
        const bool own = c == 0 && t < n;
        double px[3] = {0.0, 0.0, 0.0}, pv[3] = {0.0, 0.0, 0.0}, pm = 0.0, acc[3] = {0.0, 0.0, 0.0};
        if (own) {
            for (int k = 0; k < D; ++k) {
                px[k] = a.x[k][o + t];
                pv[k] = a.v[k][o + t];
            }
            pm = a.m[o + t];
        }
        __syncthreads();                              // the previous system's last reads of sp / sa
        if (c == 0) sp[t] = make_double4(px[0], px[1], px[2], pm);
        auto accel = [&]() {
            __syncthreads();                          // positions written
            const double4 me = sp[t];
            double ax = 0.0, ay = 0.0, az = 0.0;
            if (t < n) {
                for (int j = c; j < n; j += S) {
                    const double4 sj = sp[j];
                    const double dx = sj.x - me.x, dy = sj.y - me.y;
                    const double dz = (D == 3) ? sj.z - me.z : 0.0;
                    double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, a.eps2)));
                    const bool self = j == t;
                    if (self) r2 = 1.0;
                    const double inv = rsqrt(r2);
                    const double f = self ? 0.0 : ((G * sj.w * inv) * inv) * inv;
                    ax = fma(f, dx, ax);
                    ay = fma(f, dy, ay);
                    if (D == 3) az = fma(f, dz, az);
                }
            }
            sa[c][0][t] = ax;
            sa[c][1][t] = ay;
            sa[c][2][t] = az;
            __syncthreads();                          // partials written
            if (c == 0) {
                double r0 = 0.0, r1 = 0.0, r2 = 0.0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    r0 += sa[k][0][t];
                    r1 += sa[k][1][t];
                    r2 += sa[k][2][t];
                }
                acc[0] = r0;
                acc[1] = r1;
                acc[2] = r2;
            }
        };
        accel();
        for (int st = 0; st < a.steps; ++st) {
#pragma unroll
            for (int w = 0; w < 3; ++w) {
                const double h = wd[w] * dt;
                const double hh = 0.5 * h;
                if (c == 0) {
                    for (int k = 0; k < D; ++k) {
                        pv[k] += acc[k] * hh;
                        px[k] += pv[k] * h;
                    }
                }
                __syncthreads();                      // everyone is done reading sp
                if (c == 0) sp[t] = make_double4(px[0], px[1], px[2], pm);
                accel();
                if (c == 0)
                    for (int k = 0; k < D; ++k) pv[k] += acc[k] * hh;
            }
        }
        if (own)
            for (int k = 0; k < D; ++k) {
                a.x[k][o + t] = px[k];
                a.v[k][o + t] = pv[k];
            }
    }
}

template <int D>
void* pick_blk(int NT, int S) {
#define SSS_BLK(nt, s) if (NT == nt && S == s) return (void*)k_batched_blk<D, nt, s>;
    SSS_BLK(16, 4) SSS_BLK(16, 8) SSS_BLK(32, 2) SSS_BLK(32, 4) SSS_BLK(32, 8) SSS_BLK(64, 2) SSS_BLK(64, 4)
    SSS_BLK(64, 8)
#undef SSS_BLK
    return nullptr;
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
    // team > 32: a block per system, NT = 16, 32 or 64 targets (by max_n) x S = team / NT source chunks
    const bool blk = team > 32;
    const int nt = max_n <= 16 ? 16 : (max_n <= 32 ? 32 : 64);
    void* fn = nullptr;
    if (blk) {
        if (per_lane == 1 && team % nt == 0)
            fn = (dim == 3) ? pick_blk<3>(nt, team / nt) : pick_blk<2>(nt, team / nt);
    } else {
        fn = (dim == 3) ? pick<3>(team, per_lane) : pick<2>(team, per_lane);
    }
    if (!fn) return sss_set_err(ctx, SSS_ERR_ARG, "unsupported team mapping T=%d B=%d", team, per_lane);
    if (max_n < 1 || max_n > team * per_lane || (blk && max_n > 64))
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
        blocks = blk ? n_list : (int)((teams * team + 127) / 128);
        if (blocks < 1) blocks = 1;
    }
    void* args[] = {&a};
    SSS_CUDA_TRY(ctx, cudaLaunchKernel(fn, dim3(blocks), dim3(blk ? team : 128), args, 0, (cudaStream_t)stream));
    return SSS_OK;
}
