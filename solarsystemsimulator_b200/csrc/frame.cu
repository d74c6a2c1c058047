// Few-massive-body integrator for sm_100a: replaces `frame_kernel`
// (reference backend/nbody_kernel.py:97-560) for one GPU.
//
// Physics (unchanged from the reference): massive bodies (M <= 64) act on
// each other and on the asteroids; asteroids act back on the massive bodies
// (back-reaction) but not on each other; softening SOFTENING is added to r^2.
// Per raster sample the time advances in substeps dtH, the smallest massive
// pair encounter time / 20 (capped at max_sub_dt, floored at max_sub_dt/1000).
// Calm asteroids and massive bodies take one 4th-order Yoshida step (three
// velocity-Verlet stages) per dtH; "hot" asteroids (an encounter time / 20
// below dtH) integrate the segment in a private adaptive loop against
// linearly interpolated massive positions, recording contact times and
// sub-samples on the raster.
//
// Layout on the GPU: every CTA keeps a replica of the massive state in shared
// memory and integrates it itself. All CTAs compute bit-identical massive
// trajectories because every reduction (back-reaction sums, pair minima,
// massive-pair sums) has a fixed order. Hence:
// * massless asteroids (no back-reaction): no grid-wide synchronisation at
//   all — each CTA runs the whole launch for its asteroid chunk;
// * asteroids with mass: one grid barrier per Yoshida stage (after each CTA
//   has written its back-reaction partial), then every CTA adds all partials
//   in ascending CTA order. The barrier is a bounded spin (SSS_ERR_TIMEOUT)
//   under a cooperative launch, which guarantees co-residency.
// The reference instead runs ~8 grid.syncs per substep with a serial thread 0
// for the massive bodies and float atomics for the back-reaction.

#include "sss_internal.cuh"

namespace {

constexpr int FR_NT = 256;
constexpr int FR_WARPS = FR_NT / 32;
constexpr int M_MAX = SSS_M_MAX;
// A hot asteroid's fine loop runs on FG lanes, lane l taking the massive
// bodies k = l, l + FG, ...; the CTA's hot asteroids are listed HOT_SPAN
// asteroids at a time and handed to its FR_NT / FG lane groups on demand.
constexpr int FG = 8;
constexpr int HOT_SPAN = 2048;

struct FrameArgs {
    double* ax[3];            // asteroid positions [n_ast] per dimension
    double* av[3];            // velocities
    double* aacc[3];          // accelerations (work)
    const double* am;
    const unsigned char* avis;
    const double* arad;
    const int64_t* aidx;      // original body index of each asteroid
    unsigned char* hot;       // [n_ast] work
    double* mx[3];            // massive state [M] (read at launch, written back)
    double* mv[3];
    const double* mm;
    const unsigned char* mvis;
    const double* mrad;
    const int64_t* midx;
    int n_ast, M;
    int64_t n_total;
    double G, soft, dt_raster, max_sub_dt, w1, w0;
    int K, max_sub_steps, m_sub, massless;
    float* snap;              // [K][2D][n_total] original order
    float* sub_pos;           // [K][m_sub][D][n_ast]
    unsigned char* sub_n;     // [K][n_ast]
    float* hit_t;             // [n_ast], < 0: none
    int* hit_m;               // [n_ast] compact massive index
    double* part;             // [2][grid][3][M_MAX] back-reaction partials
    unsigned* gbar;           // [2] arrival count, generation
    int* status;
    int* guard_out;           // substeps used (written by CTA 0)
    int fine_guard;           // iteration limit of a hot asteroid's fine loop
    int pair_f32;             // 1: asteroid x massive pair forces in f32 (calm asteroids, back-reaction)
    uint64_t wait_ns;         // limit of a grid-barrier wait
};

struct FrameShared {
    double mx[3][M_MAX], mv[3][M_MAX], macc[3][M_MAX], mnew[3][M_MAX], mx0[3][M_MAX];
    double mm[M_MAX], mrad[M_MAX];
    double bk[3][M_MAX];
    double red[FR_WARPS];
    double dtH, rem;
    int done, guard, abort_;
    int hl[HOT_SPAN];         // hot asteroids of the current span
    int hn, hgrab;            // their count, the next one to hand out
    unsigned char mvis[M_MAX];
};

// Bounded grid barrier (cooperative launch only).
__device__ bool grid_sync(const FrameArgs& a, FrameShared& s) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = a.gbar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(a.gbar, 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(a.gbar, 0u);
            __threadfence();
            atomicAdd(a.gbar + 1, 1u);
        } else {
            const uint64_t t0 = sss_globaltimer();
            while (*vgen == gen) {
                if (sss_globaltimer() - t0 > a.wait_ns) {
                    atomicExch(a.status, SSS_ERR_TIMEOUT);
                    s.abort_ = 1;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s.abort_ == 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void chunk_of(int n, int& lo, int& hi) {
    const int per = (n + (int)gridDim.x - 1) / (int)gridDim.x;
    lo = min(n, (int)blockIdx.x * per);
    hi = min(n, lo + per);
}

// Acceleration of a body at p from the visible massive bodies at `mpos`.
// Same expression order as the reference: f = G/(r2 sqrt r2); a += f m dx.
template <int D>
__device__ __forceinline__ void massive_field(const FrameShared& s, const double (*mpos)[M_MAX], int M,
                                              double G, double soft, const double* p, double* acc) {
    for (int c = 0; c < D; ++c) acc[c] = 0.0;
    for (int k = 0; k < M; ++k) {
        if (!s.mvis[k]) continue;
        double dx[3], r2 = 0.0;
        for (int c = 0; c < D; ++c) { dx[c] = mpos[c][k] - p[c]; r2 += dx[c] * dx[c]; }
        r2 += soft;
        const double f = G / (r2 * sqrt(r2));
        for (int c = 0; c < D; ++c) acc[c] += f * s.mm[k] * dx[c];
    }
}

// The f32-pair form (the asteroid-cloud configuration: FP32 pair forces with
// FP64 state): the offset formed in f64 and rounded to f32, r^2, the f32
// reciprocal square root and the pair factor in f32, the sum in f64.
template <int D>
__device__ __forceinline__ void massive_field_f32(const FrameShared& s, const double (*mpos)[M_MAX], int M,
                                                  double G, double soft, const double* p, double* acc) {
    for (int c = 0; c < D; ++c) acc[c] = 0.0;
    const float Gf = (float)G, sf = (float)soft;
    for (int k = 0; k < M; ++k) {
        if (!s.mvis[k]) continue;
        float dx[3], r2 = sf;
        for (int c = 0; c < D; ++c) { dx[c] = (float)(mpos[c][k] - p[c]); r2 = fmaf(dx[c], dx[c], r2); }
        const float inv = rsqrtf(r2);
        const float f = Gf * (float)s.mm[k] * inv * inv * inv;
        for (int c = 0; c < D; ++c) acc[c] += (double)(f * dx[c]);
    }
}

// massive_field on the FG lanes of a group (mask gmask, this lane gl): lane
// gl forms the pair factor f m and the offset of bodies k = k0 + gl, then
// every lane adds the terms in ascending k, so each lane holds the sum in the
// serial order of massive_field. INTERP: the massive positions interpolated
// between mx0 and mx at fraction al.
template <int D, bool INTERP>
__device__ __forceinline__ void field_grp(const FrameShared& s, int M, double G, double soft, double al,
                                          const double* p, double* acc, int gl, unsigned gmask) {
    for (int c = 0; c < D; ++c) acc[c] = 0.0;
    for (int k0 = 0; k0 < M; k0 += FG) {
        const int k = k0 + gl;
        double fm = 0.0, dx[3] = {0.0, 0.0, 0.0};
        if (k < M && s.mvis[k]) {
            double r2 = 0.0;
            for (int c = 0; c < D; ++c) {
                double mi;
                if constexpr (INTERP) mi = s.mx0[c][k] + (s.mx[c][k] - s.mx0[c][k]) * al;
                else mi = s.mx[c][k];
                dx[c] = mi - p[c];
                r2 += dx[c] * dx[c];
            }
            r2 += soft;
            const double f = G / (r2 * sqrt(r2));
            fm = f * s.mm[k];
        }
        const int kn = min(FG, M - k0);
        for (int j = 0; j < kn; ++j) {
            if (!s.mvis[k0 + j]) continue;
            const double fj = __shfl_sync(gmask, fm, j, FG);
            for (int c = 0; c < D; ++c) acc[c] += fj * __shfl_sync(gmask, dx[c], j, FG);
        }
    }
}

// Back-reaction of this CTA's visible asteroids on every massive body:
// warp w owns bodies k = w, w+8, ...; lanes run over the asteroids in a fixed
// order and the warp sum is a fixed butterfly -> partial in a.part[slot].
template <int D>
__device__ void back_partial(const FrameArgs& a, const FrameShared& s, int lo, int hi, int slot) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* out = a.part + ((size_t)slot * gridDim.x + blockIdx.x) * 3 * M_MAX;
    for (int k = warp; k < a.M; k += FR_WARPS) {
        double b[3] = {0.0, 0.0, 0.0};
        if (s.mvis[k]) {
            for (int i = lo + lane; i < hi; i += 32) {
                if (!a.avis[i]) continue;
                if (a.pair_f32) {
                    float dx[3], r2 = (float)a.soft;
                    for (int c = 0; c < D; ++c) {
                        dx[c] = (float)(s.mx[c][k] - a.ax[c][i]);
                        r2 = fmaf(dx[c], dx[c], r2);
                    }
                    const float inv = rsqrtf(r2);
                    const float f = (float)a.G * (float)a.am[i] * inv * inv * inv;
                    for (int c = 0; c < D; ++c) b[c] -= (double)(f * dx[c]);
                    continue;
                }
                double dx[3], r2 = 0.0;
                for (int c = 0; c < D; ++c) { dx[c] = s.mx[c][k] - a.ax[c][i]; r2 += dx[c] * dx[c]; }
                r2 += a.soft;
                const double f = a.G / (r2 * sqrt(r2));
                for (int c = 0; c < D; ++c) b[c] += -f * a.am[i] * dx[c];
            }
        }
        for (int c = 0; c < D; ++c) {
            const double t = warp_sum(b[c]);
            if (lane == 0) __stcg(out + c * M_MAX + k, t);
        }
    }
}

// bk[c][k] = sum over CTAs (ascending) of the partials in `slot`.
template <int D>
__device__ void back_sum(const FrameArgs& a, FrameShared& s, int slot) {
    for (int t = threadIdx.x; t < D * a.M; t += blockDim.x) {
        const int c = t / a.M, k = t - c * a.M;
        double acc = 0.0;
        const double* base = a.part + (size_t)slot * gridDim.x * 3 * M_MAX + c * M_MAX + k;
        for (unsigned b = 0; b < gridDim.x; ++b) acc += __ldcg(base + (size_t)b * 3 * M_MAX);
        s.bk[c][k] = acc;
    }
}

// mnew = bk + sum over visible massive pairs (one warp per body, lanes over
// partners, fixed butterfly order).
template <int D>
__device__ void massive_accel(const FrameArgs& a, FrameShared& s) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < a.M; i += FR_WARPS) {
        double acc[3] = {0.0, 0.0, 0.0};
        if (s.mvis[i]) {
            for (int j = lane; j < a.M; j += 32) {
                if (j == i || !s.mvis[j]) continue;
                double dx[3], r2 = 0.0;
                for (int c = 0; c < D; ++c) { dx[c] = s.mx[c][j] - s.mx[c][i]; r2 += dx[c] * dx[c]; }
                r2 += a.soft;
                const double f = a.G / (r2 * sqrt(r2));
                for (int c = 0; c < D; ++c) acc[c] += f * s.mm[j] * dx[c];
            }
        }
        for (int c = 0; c < D; ++c) {
            const double t = warp_sum(acc[c]);
            if (lane == 0) s.mnew[c][i] = s.bk[c][i] + t;
        }
    }
}

// Smallest massive-pair encounter time / 20 (pairs spread over the CTA,
// min-reduced: order-independent).
template <int D>
__device__ double pair_dt(const FrameArgs& a, FrameShared& s) {
    double best = a.max_sub_dt;
    const int M = a.M;
    for (int t = threadIdx.x; t < M * M; t += blockDim.x) {
        const int i = t / M, j = t - i * M;
        if (j <= i || !s.mvis[i] || !s.mvis[j]) continue;
        double d2 = 0.0, v2 = 0.0;
        for (int c = 0; c < D; ++c) {
            const double dx = s.mx[c][j] - s.mx[c][i], dv = s.mv[c][j] - s.mv[c][i];
            d2 += dx * dx;
            v2 += dv * dv;
        }
        double dist = sqrt(d2);
        if (dist < 1e-12) dist = 1e-12;
        const double vrel = sqrt(v2);
        if (vrel > 1e-9) {
            const double te = dist / vrel / 20.0;
            if (te < best) best = te;
        }
    }
    for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) s.red[threadIdx.x >> 5] = best;
    __syncthreads();
    double r = s.red[0];
    for (int w = 1; w < FR_WARPS; ++w) r = fmin(r, s.red[w]);
    __syncthreads();
    return r;
}

// Hot asteroid i: private adaptive Yoshida over [0, dtH] (nbody_kernel.py:416-535)
// on the FG lanes of a group. The massive bodies are spread over the lanes
// (field_grp); the step size is the group minimum of the encounter times, a
// contact the first body in k order (the ballot's lowest bit). Every lane
// carries the same position, velocity and step, formed in the same order as
// the serial loop; lane 0 writes.
template <int D>
__device__ void fine_loop(const FrameArgs& a, const FrameShared& s, int i, int ks, double dtH, double tSeg0,
                          int gl, unsigned gmask) {
    const double wd[3] = {a.w1, a.w0, a.w1};
    const int gbase = (threadIdx.x & 31) & ~(FG - 1);
    double p[3], v[3];
    for (int c = 0; c < D; ++c) { p[c] = a.ax[c][i]; v[c] = a.av[c][i]; }
    const double sgn = dtH >= 0.0 ? 1.0 : -1.0;
    const double span = fabs(dtH);
    const double subDt = a.m_sub > 0 ? a.dt_raster / a.m_sub : 0.0;
    const double rad = a.arad[i];
    bool open = a.hit_t[i] < 0.0f;      // no contact time recorded yet
    double tau = 0.0;
    int guardF = 0;
    while (tau < span - 1e-15 && guardF++ < a.fine_guard) {
        const double al = tau / span;
        double dtF = a.max_sub_dt;
        int first = -1, last = -1;      // bodies in contact, lowest and highest k
        // one pass over the bodies at fraction al: the encounter times, the contacts and the
        // first stage's acceleration (field_grp at tau, from the same offsets)
        double acc[3];
        for (int c = 0; c < D; ++c) acc[c] = 0.0;
        for (int k0 = 0; k0 < a.M; k0 += FG) {
            const int k = k0 + gl;
            bool touch = false;
            double fm = 0.0, dx[3] = {0.0, 0.0, 0.0};
            if (k < a.M && s.mvis[k]) {
                double d2 = 0.0, v2 = 0.0;
                for (int c = 0; c < D; ++c) {
                    const double mi = s.mx0[c][k] + (s.mx[c][k] - s.mx0[c][k]) * al;
                    dx[c] = mi - p[c];
                    const double dv = s.mv[c][k] - v[c];
                    d2 += dx[c] * dx[c];
                    v2 += dv * dv;
                }
                double dist = sqrt(d2);
                if (dist < 1e-12) dist = 1e-12;
                touch = dist <= s.mrad[k] + rad;
                const double vrel = sqrt(v2);
                if (vrel > 1e-9) {
                    const double te = dist / vrel / 20.0;
                    if (te < dtF) dtF = te;
                }
                const double r2 = d2 + a.soft;
                const double f = a.G / (r2 * sqrt(r2));
                fm = f * s.mm[k];
            }
            const unsigned b = (__ballot_sync(gmask, touch) >> gbase) & ((1u << FG) - 1u);
            if (b) {
                if (first < 0) first = k0 + __ffs(b) - 1;
                last = k0 + 31 - __clz(b);
            }
            const int kn = min(FG, a.M - k0);
            for (int j = 0; j < kn; ++j) {
                if (!s.mvis[k0 + j]) continue;
                const double fj = __shfl_sync(gmask, fm, j, FG);
                for (int c = 0; c < D; ++c) acc[c] += fj * __shfl_sync(gmask, dx[c], j, FG);
            }
        }
        for (int o = FG / 2; o > 0; o >>= 1) dtF = fmin(dtF, __shfl_xor_sync(gmask, dtF, o, FG));
        if (open && first >= 0) {
            // the serial test `hit_t < 0` per body: the first body in contact closes it,
            // unless the recorded time is itself negative (then every later body overwrites)
            const float h = (float)(ks * a.dt_raster + tSeg0 + tau);
            if (gl == 0) {
                a.hit_t[i] = h;
                a.hit_m[i] = h < 0.0f ? last : first;
            }
            open = h < 0.0f;
        }
        if (dtF < a.max_sub_dt / 1000.0) dtF = a.max_sub_dt / 1000.0;
        if (dtF > span - tau) dtF = span - tau;
        if (a.m_sub > 0) {
            const double tAbs = tSeg0 + tau;
            const int jn = (int)floor(tAbs / subDt + 1e-9) + 1;
            if (jn <= a.m_sub) {
                const double rest = jn * subDt - tAbs;
                if (rest > 0.0 && dtF > rest) dtF = rest;
            }
        }
        // the three velocity-Verlet stages; a stage's closing acceleration (same time, same
        // position) is the next stage's opening one
        double tSub = tau;
        for (int wf = 0; wf < 3; ++wf) {
            const double df = wd[wf] * dtF * sgn;
            double ncc[3];
            for (int c = 0; c < D; ++c) p[c] += v[c] * df + 0.5 * acc[c] * df * df;
            tSub += wd[wf] * dtF;
            field_grp<D, true>(s, a.M, a.G, a.soft, tSub / span, p, ncc, gl, gmask);
            for (int c = 0; c < D; ++c) {
                v[c] += 0.5 * (acc[c] + ncc[c]) * df;
                acc[c] = ncc[c];
            }
        }
        tau += dtF;
        if (a.m_sub > 0 && gl == 0) {
            const double q = (tSeg0 + tau) / subDt;
            const int j = (int)floor(q + 0.5);
            if (j >= 1 && j <= a.m_sub && fabs(q - j) < 1e-6) {
                const int64_t b = ((int64_t)ks * a.m_sub + (j - 1)) * D * a.n_ast;
                for (int c = 0; c < D; ++c) a.sub_pos[b + (int64_t)c * a.n_ast + i] = (float)p[c];
                a.sub_n[(int64_t)ks * a.n_ast + i]++;
            }
        }
    }
    double acc[3];
    field_grp<D, false>(s, a.M, a.G, a.soft, 0.0, p, acc, gl, gmask);
    if (gl == 0) {
        // the guard ran out before the interval was covered: the reference stops there silently
        // (nbody_kernel.py:424); the state keeps it, the status word records it
        if (tau < span - 1e-15) atomicCAS(a.status, SSS_OK, SSS_ERR_GUARD);
        for (int c = 0; c < D; ++c) { a.ax[c][i] = p[c]; a.av[c][i] = v[c]; a.aacc[c][i] = acc[c]; }
    }
}

// The fine loops of this CTA's hot visible asteroids in [lo, hi): listed
// HOT_SPAN asteroids at a time, each taken by the next free lane group.
template <int D>
__device__ void hot_pass(const FrameArgs& a, FrameShared& s, int lo, int hi, int ks, double dtH, double tSeg0) {
    const int gl = threadIdx.x & (FG - 1);
    const unsigned gmask = ((1u << FG) - 1u) << ((threadIdx.x & 31) & ~(FG - 1));
    for (int base = lo; base < hi; base += HOT_SPAN) {
        const int end = min(hi, base + HOT_SPAN);
        if (threadIdx.x == 0) { s.hn = 0; s.hgrab = 0; }
        __syncthreads();
        for (int i = base + (int)threadIdx.x; i < end; i += blockDim.x)
            if (a.avis[i] && a.hot[i]) s.hl[atomicAdd(&s.hn, 1)] = i;
        __syncthreads();
        const int hn = s.hn;
        for (;;) {
            int j = 0;
            if (gl == 0) j = atomicAdd(&s.hgrab, 1);
            j = __shfl_sync(gmask, j, 0, FG);
            if (j >= hn) break;
            fine_loop<D>(a, s, s.hl[j], ks, dtH, tSeg0, gl, gmask);
        }
        __syncthreads();
    }
    __syncthreads();
}

// Back-reaction sums for the current asteroid positions into s.bk (all
// CTAs identical). Returns false if the grid barrier timed out.
template <int D>
__device__ bool back_reaction(const FrameArgs& a, FrameShared& s, int lo, int hi, int& slot) {
    if (a.massless) {
        for (int t = threadIdx.x; t < 3 * M_MAX; t += blockDim.x) (&s.bk[0][0])[t] = 0.0;
        __syncthreads();
        return true;
    }
    back_partial<D>(a, s, lo, hi, slot);
    if (!grid_sync(a, s)) return false;
    back_sum<D>(a, s, slot);
    slot ^= 1;
    __syncthreads();
    return true;
}

template <int D>
__global__ void __launch_bounds__(FR_NT) k_frame(const FrameArgs a) {
    __shared__ FrameShared s;
    const int tid = threadIdx.x;
    int lo, hi;
    chunk_of(a.n_ast, lo, hi);
    if (tid == 0) { s.abort_ = 0; s.guard = 0; }
    for (int k = tid; k < a.M; k += blockDim.x) {
        for (int c = 0; c < D; ++c) { s.mx[c][k] = a.mx[c][k]; s.mv[c][k] = a.mv[c][k]; }
        s.mm[k] = a.mm[k];
        s.mrad[k] = a.mrad[k];
        s.mvis[k] = a.mvis[k];
    }
    __syncthreads();
    int slot = 0;

    // initial accelerations (nbody_kernel.py:151-216)
    for (int i = lo + tid; i < hi; i += blockDim.x) {
        double p[3], acc[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < D; ++c) p[c] = a.ax[c][i];
        if (a.avis[i]) {
            if (a.pair_f32) massive_field_f32<D>(s, s.mx, a.M, a.G, a.soft, p, acc);
            else massive_field<D>(s, s.mx, a.M, a.G, a.soft, p, acc);
        }
        for (int c = 0; c < D; ++c) a.aacc[c][i] = acc[c];
    }
    if (!back_reaction<D>(a, s, lo, hi, slot)) return;
    massive_accel<D>(a, s);
    __syncthreads();
    for (int k = tid; k < a.M; k += blockDim.x)
        for (int c = 0; c < D; ++c) s.macc[c][k] = s.mnew[c][k];
    __syncthreads();

    const double wd[3] = {a.w1, a.w0, a.w1};
    for (int ks = 0; ks < a.K; ++ks) {
        if (tid == 0) { s.rem = a.dt_raster; s.done = 0; }
        if (a.m_sub > 0)
            for (int i = lo + tid; i < hi; i += blockDim.x) a.sub_n[(int64_t)ks * a.n_ast + i] = 0;
        __syncthreads();
        for (;;) {
            // dtH (nbody_kernel.py:247-275)
            const double dmin = pair_dt<D>(a, s);
            if (tid == 0) {
                if (s.rem <= 1e-12 || s.guard++ >= a.max_sub_steps) {
                    // a raster left unfinished by the substep guard (nbody_kernel.py:248-250)
                    if (s.rem > 1e-12) atomicCAS(a.status, SSS_OK, SSS_ERR_GUARD);
                    s.done = 1;
                } else {
                    double dtH = dmin;
                    if (dtH < a.max_sub_dt / 1000.0) dtH = a.max_sub_dt / 1000.0;
                    if (dtH > s.rem) dtH = s.rem;
                    s.dtH = dtH;
                    s.rem -= dtH;
                }
            }
            __syncthreads();
            if (s.done) break;
            const double dtH = s.dtH;
            // hot classification (:283-301)
            for (int i = lo + tid; i < hi; i += blockDim.x) {
                unsigned char h = 0;
                if (a.avis[i]) {
                    for (int k = 0; k < a.M && !h; ++k) {
                        if (!s.mvis[k]) continue;
                        double d2 = 0.0, v2 = 0.0;
                        for (int c = 0; c < D; ++c) {
                            const double dx = s.mx[c][k] - a.ax[c][i], dv = s.mv[c][k] - a.av[c][i];
                            d2 += dx * dx;
                            v2 += dv * dv;
                        }
                        double dist = sqrt(d2);
                        if (dist < 1e-12) dist = 1e-12;
                        const double vrel = sqrt(v2);
                        if (vrel > 1e-9 && dist / vrel / 20.0 < dtH) h = 1;
                    }
                }
                a.hot[i] = h;
            }
            for (int k = tid; k < a.M; k += blockDim.x)
                for (int c = 0; c < D; ++c) s.mx0[c][k] = s.mx[c][k];
            __syncthreads();

            for (int w = 0; w < 3; ++w) {
                const double dt = wd[w] * dtH;
                // phase A: positions of calm asteroids and massive bodies (:317-331)
                for (int i = lo + tid; i < hi; i += blockDim.x) {
                    if (!a.avis[i] || a.hot[i]) continue;
                    for (int c = 0; c < D; ++c) a.ax[c][i] += a.av[c][i] * dt + 0.5 * a.aacc[c][i] * dt * dt;
                }
                for (int k = tid; k < a.M; k += blockDim.x) {
                    if (!s.mvis[k]) continue;
                    for (int c = 0; c < D; ++c) s.mx[c][k] += s.mv[c][k] * dt + 0.5 * s.macc[c][k] * dt * dt;
                }
                __syncthreads();
                // phase B: asteroid forces + velocities of calm asteroids (:343-362)
                for (int i = lo + tid; i < hi; i += blockDim.x) {
                    if (!a.avis[i]) continue;
                    double p[3], acc[3];
                    for (int c = 0; c < D; ++c) p[c] = a.ax[c][i];
                    if (a.pair_f32 && !a.hot[i]) massive_field_f32<D>(s, s.mx, a.M, a.G, a.soft, p, acc);
                    else massive_field<D>(s, s.mx, a.M, a.G, a.soft, p, acc);
                    if (!a.hot[i]) {
                        for (int c = 0; c < D; ++c) {
                            a.av[c][i] += 0.5 * (a.aacc[c][i] + acc[c]) * dt;
                            a.aacc[c][i] = acc[c];
                        }
                    }
                }
                // back-reaction of all visible asteroids (hot ones at their segment start)
                if (!back_reaction<D>(a, s, lo, hi, slot)) return;
                // phase C: massive accelerations and velocities (:377-399)
                massive_accel<D>(a, s);
                __syncthreads();
                for (int k = tid; k < a.M; k += blockDim.x) {
                    for (int c = 0; c < D; ++c) {
                        if (s.mvis[k]) s.mv[c][k] += 0.5 * (s.macc[c][k] + s.mnew[c][k]) * dt;
                        s.macc[c][k] = s.mnew[c][k];
                    }
                }
                __syncthreads();
            }
            // private fine loop of the hot asteroids (:416-535)
            hot_pass<D>(a, s, lo, hi, ks, dtH, a.dt_raster - s.rem - dtH);
        }
        // snapshot of this raster sample, original body order (:540-557)
        float* row = a.snap + (int64_t)ks * 2 * D * a.n_total;
        for (int i = lo + tid; i < hi; i += blockDim.x) {
            const int64_t o = a.aidx[i];
            for (int c = 0; c < D; ++c) {
                row[(int64_t)c * a.n_total + o] = (float)a.ax[c][i];
                row[(int64_t)(D + c) * a.n_total + o] = (float)a.av[c][i];
            }
        }
        if (blockIdx.x == 0) {
            for (int k = tid; k < a.M; k += blockDim.x) {
                const int64_t o = a.midx[k];
                for (int c = 0; c < D; ++c) {
                    row[(int64_t)c * a.n_total + o] = (float)s.mx[c][k];
                    row[(int64_t)(D + c) * a.n_total + o] = (float)s.mv[c][k];
                }
            }
        }
        __syncthreads();
    }
    if (blockIdx.x == 0) {
        for (int k = tid; k < a.M; k += blockDim.x)
            for (int c = 0; c < D; ++c) { a.mx[c][k] = s.mx[c][k]; a.mv[c][k] = s.mv[c][k]; }
        if (tid == 0) *a.guard_out = s.guard;
    }
}

// Self-test of the bounded grid barrier: CTA 1 leaves without arriving, so
// CTA 0's wait runs out after a.wait_ns and records SSS_ERR_TIMEOUT.
__global__ void k_frame_barrier_selftest(const FrameArgs a) {
    __shared__ FrameShared s;
    if (threadIdx.x == 0) s.abort_ = 0;
    __syncthreads();
    if (blockIdx.x != 0) return;
    grid_sync(a, s);
}

// Scatter updates at original indices into the resident state:
// mode 0 = set x,v; 1 = add to x,v; 2 = set x,v and mass; vals [m][2D(+1)].
struct ScatterPtrs {
    double* ax[3];
    double* av[3];
    double* mx[3];
    double* mv[3];
    double* am;
    double* mm;
};

__global__ void k_frame_scatter(const ScatterPtrs p, const int64_t* __restrict__ slot,
                                const double* __restrict__ vals, int m, int dim, int mode) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int64_t sl = slot[t];          // >= 0: asteroid sl; < 0: massive -sl-1
    const int w = 2 * dim + (mode == 2 ? 1 : 0);
    const double* v = vals + (int64_t)t * w;
    const bool ast = sl >= 0;
    const int64_t k = ast ? sl : -sl - 1;
    for (int c = 0; c < dim; ++c) {
        double* X = ast ? p.ax[c] : p.mx[c];
        double* V = ast ? p.av[c] : p.mv[c];
        if (mode == 1) { X[k] += v[c]; V[k] += v[dim + c]; }
        else { X[k] = v[c]; V[k] = v[dim + c]; }
    }
    if (mode == 2) (ast ? p.am : p.mm)[k] = v[2 * dim];
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" int sss_frame_launch(sss_ctx* ctx, const sss_frame_state* st, double dt_raster, int k, int m_sub,
                                float* snap, float* sub_pos, unsigned char* sub_n, float* hit_t, int* hit_m,
                                int* guard_used, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!st) return sss_set_err(ctx, SSS_ERR_ARG, "NULL state");
    if (st->dim != 2 && st->dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3");
    if (st->M < 0 || st->M > SSS_M_MAX)
        return sss_set_err(ctx, SSS_ERR_TOO_MANY_MASSIVE, "zu viele massive Koerper: %d > %d", st->M, SSS_M_MAX);
    if (st->n_ast < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative asteroid count");
    if (k < 1 || k > SSS_K_MAX) return sss_set_err(ctx, SSS_ERR_ARG, "k ausserhalb 1..%d: %d", SSS_K_MAX, k);
    if (m_sub < 0 || m_sub > SSS_SUB_SAMPLES_MAX)
        return sss_set_err(ctx, SSS_ERR_ARG, "m_sub ausserhalb 0..%d: %d", SSS_SUB_SAMPLES_MAX, m_sub);
    if (!snap || !guard_used || (st->n_ast > 0 && (!hit_t || !hit_m)) ||
        (m_sub > 0 && st->n_ast > 0 && (!sub_pos || !sub_n)))
        return sss_set_err(ctx, SSS_ERR_ARG, "NULL output buffer");
    if (!(dt_raster == dt_raster)) return sss_set_err(ctx, SSS_ERR_ARG, "dt is NaN");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int D = st->dim;

    FrameArgs a;
    memset(&a, 0, sizeof(a));
    for (int c = 0; c < 3; ++c) {
        a.ax[c] = st->ast_x[c];
        a.av[c] = st->ast_v[c];
        a.aacc[c] = st->ast_acc[c];
        a.mx[c] = st->mas_x[c];
        a.mv[c] = st->mas_v[c];
    }
    a.am = st->ast_m;
    a.avis = st->ast_vis;
    a.arad = st->ast_r;
    a.aidx = st->ast_idx;
    a.hot = st->ast_hot;
    a.mm = st->mas_m;
    a.mvis = st->mas_vis;
    a.mrad = st->mas_r;
    a.midx = st->mas_idx;
    a.n_ast = (int)st->n_ast;
    a.M = st->M;
    a.n_total = st->n_ast + st->M;
    a.G = st->G;
    a.soft = st->softening;
    a.dt_raster = dt_raster;
    a.max_sub_dt = st->max_sub_dt;
    a.max_sub_steps = st->max_sub_steps;
    a.w1 = st->w1;
    a.w0 = st->w0;
    a.K = k;
    a.m_sub = m_sub;
    a.massless = st->massless_asteroids;
    a.snap = snap;
    a.sub_pos = sub_pos;
    a.sub_n = sub_n;
    a.hit_t = hit_t;
    a.hit_m = hit_m;
    a.status = ctx->d_status;
    a.guard_out = guard_used;
    a.fine_guard = st->fine_guard > 0 ? st->fine_guard : SSS_FINE_GUARD;
    a.pair_f32 = st->pair_f32 ? 1 : 0;
    a.wait_ns = SSS_WAIT_LIMIT_NS;

    void* fn = (D == 3) ? (void*)k_frame<3> : (void*)k_frame<2>;
    int per_sm = 0;
    SSS_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, FR_NT, 0));
    if (per_sm < 1) return sss_set_err(ctx, SSS_ERR_CUDA, "frame kernel does not fit on an SM");
    const int need = (int)((st->n_ast + FR_NT - 1) / FR_NT);
    int grid = need < 1 ? 1 : need;
    const int cap = per_sm * ctx->num_sms;
    if (grid > cap) grid = cap;
    void* args[] = {&a};
    if (a.massless) {
        SSS_CUDA_TRY(ctx, cudaLaunchKernel(fn, dim3(grid), dim3(FR_NT), args, 0, s));
        return SSS_OK;
    }
    // asteroids with mass: back-reaction partials + bounded grid barrier
    const size_t part_bytes = (size_t)2 * grid * 3 * M_MAX * sizeof(double);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, part_bytes + 256, &scr);
    if (rc) return rc;
    a.part = (double*)scr;
    a.gbar = (unsigned*)((char*)scr + part_bytes);
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(a.gbar, 0, 2 * sizeof(unsigned), s));
    SSS_CUDA_TRY(ctx, cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(FR_NT), args, 0, s));
    return SSS_OK;
}

extern "C" int sss_frame_scatter(sss_ctx* ctx, const sss_frame_state* st, const int64_t* slot,
                                 const double* vals, int m, int mode, void* stream) {
    if (!ctx) return SSS_ERR_ARG;
    if (!st || (m > 0 && (!slot || !vals))) return sss_set_err(ctx, SSS_ERR_ARG, "NULL argument");
    if (mode < 0 || mode > 2) return sss_set_err(ctx, SSS_ERR_ARG, "mode must be 0, 1 or 2");
    if (st->dim != 2 && st->dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3");
    if (m <= 0) return SSS_OK;
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    ScatterPtrs p;
    for (int c = 0; c < 3; ++c) {
        p.ax[c] = st->ast_x[c];
        p.av[c] = st->ast_v[c];
        p.mx[c] = st->mas_x[c];
        p.mv[c] = st->mas_v[c];
    }
    p.am = st->ast_m;
    p.mm = st->mas_m;
    k_frame_scatter<<<(m + 127) / 128, 128, 0, (cudaStream_t)stream>>>(p, slot, vals, m, st->dim, mode);
    SSS_LAUNCH_CHECK(ctx, "k_frame_scatter launch");
    return SSS_OK;
}

// Runs the frame kernel's grid barrier with one CTA that never arrives (see
// k_frame_barrier_selftest); the wait gives up after limit_s seconds.
int sss_frame_barrier_selftest(sss_ctx* ctx, double limit_s, cudaStream_t s) {
    void* scr = nullptr;
    int rc = sss_scratch(ctx, 256, &scr);
    if (rc) return rc;
    FrameArgs a;
    memset(&a, 0, sizeof(a));
    a.gbar = (unsigned*)scr;
    a.status = ctx->d_status;
    a.wait_ns = (uint64_t)(limit_s * 1e9);
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(a.gbar, 0, 2 * sizeof(unsigned), s));
    k_frame_barrier_selftest<<<2, FR_NT, 0, s>>>(a);
    SSS_LAUNCH_CHECK(ctx, "k_frame_barrier_selftest");
    return SSS_OK;
}
