// All-pairs Plummer self-gravity for sm_100a.
//
// Replaces the tiled force loop `beschleunigung` and the KDK step loop of
// `selfgrav_kernel` (reference backend/selfgrav_kernel.py:222-420).
//
// Work decomposition: a CTA owns a block of NT*R targets (R per thread, in
// registers) and one CHUNK of the source list. Source tiles are staged in
// shared memory by 1-D bulk async copies (cp.async.bulk + mbarrier, double
// buffered) and read back as broadcast loads. Chunks split the source sum so
// the grid has enough CTAs for an even load on 148 SMs; the chunk partials
// are added in ascending chunk order by the last CTA of each target block to
// arrive (arrival counted by one atomic per target block, no spinning), and
// that CTA runs the integrator epilogue: closing half kick, snapshot, next
// opening half kick and drift (the Yoshida / KDK sequence fused into the
// force kernel). Within a tile each target sums its sources in ascending
// index order, tiles in ascending order, as the reference does
// (selfgrav_kernel.py:235-256).
//
// Equal-mass tiles: when every source of a tile has the same Gm, the pair
// loop drops the mass multiply and the tile's sum is scaled by Gm once when
// it is folded into the accumulator (detected per tile, automatically).
//
// f64 path: every operation in f64; r^-3 from an f32 seed refined in f64.
// Mixed path: sources are pre-shifted per tile to the tile's bounding-box
// centre and rounded to f32; each target's offset to the centre is formed
// in f64 and rounded once per tile, so the f32 pair difference is a
// difference of small numbers. f32 pair terms are summed over sub-tiles of
// MIX_SUB sources and folded into f64 accumulators. The f32 arithmetic is
// issued as packed f32x2 instructions (two targets per instruction).

#include "allpairs.cuh"

#include <pthread.h>

namespace {

// f64 kernel: 2 targets per thread, 64 registers, 4 CTAs (32 warps) per SM
constexpr int F64_NT = 256;
constexpr int F64_R = 2;
constexpr int F64_TS = 512;     // sources per shared-memory tile (16 KiB)
constexpr int F64_MINB = 4;
constexpr int F64_UNROLL = 4;

// mixed kernel: 8 targets per thread (4 packed pairs), 2 CTAs per SM
constexpr int MIX_NT = 128;
constexpr int MIX_R = 8;
constexpr int MIX_TS = 512;     // sources per tile (32 B each, duplicated: 16 KiB)
constexpr int MIX_SUB = 128;    // f32 partial-sum length before the f64 fold
constexpr int MIX_MINB = 2;

constexpr int WAVES = 16;       // target number of CTA waves per evaluation

// r2 below this is outside the integer-seeded rsqrt's range (2^-126)
constexpr double kIseedMinR2 = 1.1754943508222875e-38;

using sss_ap::Epi;
using sss_ap::epilogue;

struct ForceArgs {
    const double4* src;      // f64 path: sources
    const float4* srcf;      // mixed path: tile-shifted, duplicated f32 sources
    const double4* centers;  // mixed path: tile centres, .w = common Gm or NaN
    int64_t n_src;
    const double4* tgt;
    int64_t n_tgt;
    double eps2;
    int n_tiles;
    int n_chunks;
    int tiles_per_chunk;
    double4* part;           // [n_chunks][n_tgt] partial sums (n_chunks > 1)
    unsigned* counters;      // [n_target_blocks]
    int* status;
    Epi epi;
};

// Chunk partial -> (last arriving CTA) fixed-order sum -> epilogue.
template <int D, int R, int NT>
__device__ __forceinline__ void finish_block(const ForceArgs& a, int tb, int ch,
                                             const double (&ax)[R], const double (&ay)[R],
                                             const double (&az)[R]) {
    __shared__ unsigned s_last;
    const int tid = threadIdx.x;
    const int64_t tbase = (int64_t)tb * (NT * R);
    if (a.n_chunks == 1) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int64_t i = tbase + r * NT + tid;
            if (i < a.n_tgt) epilogue<D>(a.epi, i, ax[r], ay[r], az[r], a.tgt[i]);
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t i = tbase + r * NT + tid;
        if (i < a.n_tgt) {
            double2* q = reinterpret_cast<double2*>(a.part + (int64_t)ch * a.n_tgt + i);
            __stcg(q, make_double2(ax[r], ay[r]));
            __stcg(q + 1, make_double2(az[r], 0.0));
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const unsigned prev = atomicAdd(&a.counters[tb], 1u);
        s_last = (prev == (unsigned)(a.n_chunks - 1)) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t i = tbase + r * NT + tid;
        if (i >= a.n_tgt) continue;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int c = 0; c < a.n_chunks; ++c) {
            const double2* q = reinterpret_cast<const double2*>(a.part + (int64_t)c * a.n_tgt + i);
            const double2 q0 = __ldcg(q), q1 = __ldcg(q + 1);
            sx += q0.x;
            sy += q0.y;
            sz += q1.x;
        }
        epilogue<D>(a.epi, i, sx, sy, sz, a.tgt[i]);
    }
    if (tid == 0) a.counters[tb] = 0u;  // ready for the next launch
}

// Wait (bounded) for copies still in flight after an abort, so the CTA does
// not exit while the async proxy writes its shared memory.
__device__ __noinline__ void drain_after_abort(uint64_t* bar, int issued, int consumed, int* status) {
    for (int k = consumed; k < issued; ++k) sss_mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1, status);
}

// ------------------------------------------------------------------ f64

// r2^(-3/2), times gm unless UNIT (the equal-mass tile loop scales later).
//   VAR 1: CUDA's rsqrt(double) and three multiplies
//   VAR 0: series refinement of an f32 seed formed by f64->f32 conversion
//   VAR 2: the same with the seed argument formed by integer operations
// (Measured on the benchmark shape: VAR 2 199.7 ms, VAR 0 198.8-202.6 ms,
// VAR 1 245.6 ms per evaluation; evaluating the e^2 term in f32 to save one
// f64 operation was slower, 215 ms, because of its two conversions.)
template <int VAR, bool UNIT>
__device__ __forceinline__ double rinv3(double gm, double r2) {
    if (VAR == 1) {
        const double inv = rsqrt(r2);
        return UNIT ? (inv * inv) * inv : ((gm * inv) * inv) * inv;
    }
    double c;
    if (VAR == 2) {
        // seed argument by integer re-biasing of r2's high word (valid for
        // 2^-126 <= r2 < 2^128), widened back bit by bit
        const unsigned hi = (unsigned)__double2hiint(r2);
        const float yf = sss_rsqrt_approx_f32(__uint_as_float((hi << 3) + 0x40000000u));
        const unsigned yb = __float_as_uint(yf);
        c = __hiloint2double((int)((yb >> 3) + 0x38000000u), (int)(yb << 29));
    } else {
        c = (double)sss_rsqrt_approx_f32(__double2float_rn(r2));
    }
    // c^3 (1 + 3/2 e + 15/8 e^2), e = 1 - r2 c^2 (see sss_gm_rinv3_f64)
    const double c2 = c * c;
    const double e = fma(-r2, c2, 1.0);
    const double g3 = UNIT ? c * c2 : (gm * c) * c2;
    const double p = fma(e, 1.875, 1.5);
    return fma(g3, e * p, g3);
}

template <int D, int R, int VAR, bool UNIT, int UNROLL>
__device__ __forceinline__ void tile_f64(const double4* __restrict__ s, int cnt, double eps2,
                                         const double (&px)[R], const double (&py)[R],
                                         const double (&pz)[R], double (&tx)[R], double (&ty)[R],
                                         double (&tz)[R]) {
#pragma unroll UNROLL
    for (int j = 0; j < cnt; ++j) {
        const double4 sj = s[j];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double dx = sj.x - px[r];
            const double dy = sj.y - py[r];
            double r2;
            double dz = 0.0;
            if (D == 3) {
                dz = sj.z - pz[r];
                r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
            } else {
                r2 = fma(dx, dx, fma(dy, dy, eps2));
            }
            const double f = rinv3<VAR, UNIT>(sj.w, r2);
            tx[r] = fma(f, dx, tx[r]);
            ty[r] = fma(f, dy, ty[r]);
            if (D == 3) tz[r] = fma(f, dz, tz[r]);
        }
    }
}

template <int D, int R, int NT, int TS, int VAR, int MINB, int UNROLL>
__global__ void __launch_bounds__(NT, MINB) k_force_f64(const ForceArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    double4* tiles = reinterpret_cast<double4*>(smem);
    __shared__ __align__(8) uint64_t bar[2];
    // chunk accumulators live in shared memory (touched once per tile), which
    // leaves the registers to the pair loop
    __shared__ double s_acc[3 * R][NT];

    const int S = a.n_chunks;
    const int tb = blockIdx.x / S;
    const int ch = blockIdx.x - tb * S;
    const int tid = threadIdx.x;
    const int64_t tbase = (int64_t)tb * (NT * R);

    double px[R], py[R], pz[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t i = tbase + r * NT + tid;
        const double4 p = (i < a.n_tgt) ? a.tgt[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        px[r] = p.x; py[r] = p.y; pz[r] = p.z;
        s_acc[r][tid] = 0.0;
        s_acc[R + r][tid] = 0.0;
        s_acc[2 * R + r][tid] = 0.0;
    }

    const int t_begin = ch * a.tiles_per_chunk;
    const int t_end = min(t_begin + a.tiles_per_chunk, a.n_tiles);
    const int nt = t_end - t_begin;

    if (tid == 0) {
        sss_mbar_init(&bar[0], 1);
        sss_mbar_init(&bar[1], 1);
        sss_fence_mbar_init();
    }
    __syncthreads();

    int issued = 0;
    auto issue = [&](int k) {
        const int64_t j0 = (int64_t)(t_begin + k) * TS;
        const int cnt = (int)min((int64_t)TS, a.n_src - j0);
        const unsigned bytes = (unsigned)cnt * (unsigned)sizeof(double4);
        sss_mbar_arrive_expect_tx(&bar[k & 1], bytes);
        sss_bulk_g2s(tiles + (k & 1) * TS, a.src + j0, bytes, &bar[k & 1]);
    };
    if (tid == 0) {
        issue(0);
        issued = 1;
        if (nt > 1) { issue(1); issued = 2; }
    }

    const double eps2 = a.eps2;
    int k = 0;
    for (; k < nt; ++k) {
        const int64_t j0 = (int64_t)(t_begin + k) * TS;
        const int cnt = (int)min((int64_t)TS, a.n_src - j0);
        const bool waited = sss_mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1, a.status);
        if (__syncthreads_or(!waited)) break;
        const double4* s = tiles + (k & 1) * TS;
        const double w0 = s[0].w;
        bool same = true;
        for (int j = tid; j < cnt; j += NT) same &= (s[j].w == w0);
        const bool uni = __syncthreads_and(same) != 0;
        double tx[R], ty[R], tz[R];
#pragma unroll
        for (int r = 0; r < R; ++r) { tx[r] = 0.0; ty[r] = 0.0; tz[r] = 0.0; }
        if (uni) tile_f64<D, R, VAR, true, UNROLL>(s, cnt, eps2, px, py, pz, tx, ty, tz);
        else tile_f64<D, R, VAR, false, UNROLL>(s, cnt, eps2, px, py, pz, tx, ty, tz);
        const double wt = uni ? w0 : 1.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            s_acc[r][tid] = fma(wt, tx[r], s_acc[r][tid]);
            s_acc[R + r][tid] = fma(wt, ty[r], s_acc[R + r][tid]);
            s_acc[2 * R + r][tid] = fma(wt, tz[r], s_acc[2 * R + r][tid]);
        }
        __syncthreads();
        if (tid == 0 && k + 2 < nt) { issue(k + 2); issued = k + 3; }
    }
    if (k < nt) {  // aborted on a timed-out wait
        if (tid == 0) drain_after_abort(bar, issued, k, a.status);
        return;
    }
    double ax[R], ay[R], az[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        ax[r] = s_acc[r][tid];
        ay[r] = s_acc[R + r][tid];
        az[r] = s_acc[2 * R + r][tid];
    }
    finish_block<D, R, NT>(a, tb, ch, ax, ay, az);
}

// ---------------------------------------------------------------- mixed

typedef unsigned long long f2x;   // two packed f32

__device__ __forceinline__ f2x pk2(float lo, float hi) {
    f2x r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(f2x v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2x add2(f2x a, f2x b) {
    f2x d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
    f2x d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
    f2x d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// One CTA per tile of TS sources: bounding-box centre (f64), common Gm of
// the tile (NaN if the masses differ), and every source's f32 offset from
// the centre, duplicated {x,x,y,y},{z,z,Gm,Gm} for the packed loop
// (padding entries get Gm = 0).
template <int D, int TS>
__global__ void __launch_bounds__(256) k_prep_mixed(const double4* __restrict__ src, int64_t n_src,
                                                    float4* __restrict__ out,
                                                    double4* __restrict__ centers) {
    __shared__ double red[6][8];
    __shared__ int s_diff;
    const int tile = blockIdx.x;
    const int64_t j0 = (int64_t)tile * TS;
    if (threadIdx.x == 0) s_diff = 0;
    const double w0 = src[j0].w;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    bool diff = false;
    for (int j = threadIdx.x; j < TS; j += blockDim.x) {
        const int64_t g = j0 + j;
        if (g < n_src) {
            const double4 s = src[g];
            lo[0] = fmin(lo[0], s.x); hi[0] = fmax(hi[0], s.x);
            lo[1] = fmin(lo[1], s.y); hi[1] = fmax(hi[1], s.y);
            lo[2] = fmin(lo[2], s.z); hi[2] = fmax(hi[2], s.z);
            diff |= (s.w != w0);
        }
    }
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (diff) s_diff = 1;
    if (l == 0) {
        for (int c = 0; c < 3; ++c) { red[c][w] = lo[c]; red[3 + c][w] = hi[c]; }
    }
    __syncthreads();
    double cen[3];
    for (int c = 0; c < 3; ++c) {
        double a = red[c][0], b = red[3 + c][0];
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) { a = fmin(a, red[c][q]); b = fmax(b, red[3 + c][q]); }
        cen[c] = (a <= b) ? 0.5 * (a + b) : 0.0;
    }
    if (D == 2) cen[2] = 0.0;
    if (threadIdx.x == 0)
        centers[tile] = make_double4(cen[0], cen[1], cen[2], s_diff ? __longlong_as_double(0x7ff8000000000000ll) : w0);
    for (int j = threadIdx.x; j < TS; j += blockDim.x) {
        const int64_t g = j0 + j;
        float x = 0.f, y = 0.f, z = 0.f, m = 0.f;
        if (g < n_src) {
            const double4 s = src[g];
            x = __double2float_rn(s.x - cen[0]);
            y = __double2float_rn(s.y - cen[1]);
            z = (D == 3) ? __double2float_rn(s.z - cen[2]) : 0.f;
            m = __double2float_rn(s.w);
        }
        out[2 * (j0 + j)] = make_float4(x, x, y, y);
        out[2 * (j0 + j) + 1] = make_float4(z, z, m, m);
    }
}

template <int D, int P, bool UNIT>
__device__ __forceinline__ void subtile_mixed(const ulonglong2* __restrict__ s, int js, int je, f2x eps2x,
                                              const f2x (&ox)[P], const f2x (&oy)[P], const f2x (&oz)[P],
                                              f2x (&fx)[P], f2x (&fy)[P], f2x (&fz)[P]) {
#pragma unroll 4
    for (int j = js; j < je; ++j) {
        const ulonglong2 xy = s[2 * j];
        const ulonglong2 zw = s[2 * j + 1];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const f2x dx = add2(xy.x, ox[q]);
            const f2x dy = add2(xy.y, oy[q]);
            f2x r2;
            f2x dz = 0ull;
            if (D == 3) {
                dz = add2(zw.x, oz[q]);
                r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, eps2x)));
            } else {
                r2 = fma2(dx, dx, fma2(dy, dy, eps2x));
            }
            float r0, r1;
            upk2(r2, r0, r1);
            const f2x inv = pk2(sss_rsqrt_approx_f32(r0), sss_rsqrt_approx_f32(r1));
            const f2x f = UNIT ? mul2(inv, mul2(inv, inv)) : mul2(mul2(zw.y, inv), mul2(inv, inv));
            fx[q] = fma2(f, dx, fx[q]);
            fy[q] = fma2(f, dy, fy[q]);
            if (D == 3) fz[q] = fma2(f, dz, fz[q]);
        }
    }
}

template <int D, int R, int NT, int TS, int SUB, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_force_mixed(const ForceArgs a) {
    static_assert(R % 2 == 0, "packed kernel needs an even target count");
    constexpr int P = R / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    ulonglong2* tiles = reinterpret_cast<ulonglong2*>(smem);   // [2][TS][2]
    __shared__ __align__(8) uint64_t bar[2];

    const int S = a.n_chunks;
    const int tb = blockIdx.x / S;
    const int ch = blockIdx.x - tb * S;
    const int tid = threadIdx.x;
    const int64_t tbase = (int64_t)tb * (NT * R);

    double px[R], py[R], pz[R], ax[R], ay[R], az[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t i = tbase + r * NT + tid;
        const double4 p = (i < a.n_tgt) ? a.tgt[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        px[r] = p.x; py[r] = p.y; pz[r] = p.z;
        ax[r] = 0.0; ay[r] = 0.0; az[r] = 0.0;
    }

    const int t_begin = ch * a.tiles_per_chunk;
    const int t_end = min(t_begin + a.tiles_per_chunk, a.n_tiles);
    const int nt = t_end - t_begin;

    if (tid == 0) {
        sss_mbar_init(&bar[0], 1);
        sss_mbar_init(&bar[1], 1);
        sss_fence_mbar_init();
    }
    __syncthreads();

    int issued = 0;
    constexpr unsigned kTileBytes = TS * 2 * sizeof(float4);
    const float4* srcf = a.srcf;
    auto issue = [&](int k) {
        sss_mbar_arrive_expect_tx(&bar[k & 1], kTileBytes);
        sss_bulk_g2s(tiles + (k & 1) * TS * 2, srcf + (int64_t)(t_begin + k) * TS * 2, kTileBytes, &bar[k & 1]);
    };
    if (tid == 0) {
        issue(0);
        issued = 1;
        if (nt > 1) { issue(1); issued = 2; }
    }

    const float eps2f = (float)a.eps2;
    const f2x eps2x = pk2(eps2f, eps2f);
    int k = 0;
    for (; k < nt; ++k) {
        const int tile = t_begin + k;
        const int64_t j0 = (int64_t)tile * TS;
        const int cnt = (int)min((int64_t)TS, a.n_src - j0);
        const double4 c = a.centers[tile];
        const bool uni = (c.w == c.w);   // the tile's common Gm, NaN if masses differ
        f2x ox[P], oy[P], oz[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            ox[q] = pk2(__double2float_rn(c.x - px[2 * q]), __double2float_rn(c.x - px[2 * q + 1]));
            oy[q] = pk2(__double2float_rn(c.y - py[2 * q]), __double2float_rn(c.y - py[2 * q + 1]));
            oz[q] = (D == 3) ? pk2(__double2float_rn(c.z - pz[2 * q]), __double2float_rn(c.z - pz[2 * q + 1]))
                             : pk2(0.f, 0.f);
        }
        const bool waited = sss_mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1, a.status);
        if (__syncthreads_or(!waited)) break;
        const ulonglong2* s = tiles + (k & 1) * TS * 2;
        const double wt = uni ? c.w : 1.0;
        for (int js = 0; js < cnt; js += SUB) {
            const int je = min(js + SUB, cnt);
            f2x fx[P], fy[P], fz[P];
#pragma unroll
            for (int q = 0; q < P; ++q) { fx[q] = 0ull; fy[q] = 0ull; fz[q] = 0ull; }
            if (uni) subtile_mixed<D, P, true>(s, js, je, eps2x, ox, oy, oz, fx, fy, fz);
            else subtile_mixed<D, P, false>(s, js, je, eps2x, ox, oy, oz, fx, fy, fz);
#pragma unroll
            for (int q = 0; q < P; ++q) {
                float l0, l1;
                upk2(fx[q], l0, l1);
                ax[2 * q] = fma(wt, (double)l0, ax[2 * q]);
                ax[2 * q + 1] = fma(wt, (double)l1, ax[2 * q + 1]);
                upk2(fy[q], l0, l1);
                ay[2 * q] = fma(wt, (double)l0, ay[2 * q]);
                ay[2 * q + 1] = fma(wt, (double)l1, ay[2 * q + 1]);
                if (D == 3) {
                    upk2(fz[q], l0, l1);
                    az[2 * q] = fma(wt, (double)l0, az[2 * q]);
                    az[2 * q + 1] = fma(wt, (double)l1, az[2 * q + 1]);
                }
            }
        }
        __syncthreads();
        if (tid == 0 && k + 2 < nt) { issue(k + 2); issued = k + 3; }
    }
    if (k < nt) {
        if (tid == 0) drain_after_abort(bar, issued, k, a.status);
        return;
    }
    finish_block<D, R, NT>(a, tb, ch, ax, ay, az);
}

// ------------------------------------------------------------- potential

// phi_t = -sum_s Gm_s / sqrt(|d|^2 + eps2), f64, one target per thread,
// sources through shared memory in ascending order (diagnostic path).
template <int D>
__global__ void __launch_bounds__(256) k_potential(const double4* __restrict__ src, int64_t n_src,
                                                   const double4* __restrict__ tgt, int64_t n_tgt,
                                                   double* __restrict__ phi, double eps2) {
    __shared__ double4 sh[256];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double4 p = (i < n_tgt) ? tgt[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    double acc = 0.0;
    for (int64_t j0 = 0; j0 < n_src; j0 += 256) {
        const int64_t g = j0 + threadIdx.x;
        sh[threadIdx.x] = (g < n_src) ? src[g] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        const int cnt = (int)min((int64_t)256, n_src - j0);
        for (int j = 0; j < cnt; ++j) {
            const double4 s = sh[j];
            const double dx = s.x - p.x, dy = s.y - p.y;
            double r2 = dx * dx + dy * dy + eps2;
            if (D == 3) { const double dz = s.z - p.z; r2 += dz * dz; }
            acc += s.w * rsqrt(r2);
        }
        __syncthreads();
    }
    if (i < n_tgt) phi[i] = -acc;
}

// -------------------------------------------------------------- integrate

// Opening half kick + drift of the first substep of a batch.
template <int D>
__global__ void k_open(const double4* __restrict__ pos, double4* __restrict__ pos_nxt,
                       double4* __restrict__ vel, const double4* __restrict__ acc, int64_t n,
                       double ko, double kd) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 a = acc[i];
    double4 v = vel[i];
    const double4 p = pos[i];
    v.x += a.x * ko;
    v.y += a.y * ko;
    if (D == 3) v.z += a.z * ko;
    double4 q = p;
    q.x = p.x + v.x * kd;
    q.y = p.y + v.y * kd;
    if (D == 3) q.z = p.z + v.z * kd;
    vel[i] = v;
    pos_nxt[i] = q;
}

// ---------------------------------------------------------------- host side

struct Plan {
    int n_tblocks, n_tiles, n_chunks, tiles_per_chunk;
};

Plan make_plan(int64_t n_src, int64_t n_tgt, int targets_per_block, int ts, int slots) {
    Plan p;
    p.n_tblocks = (int)((n_tgt + targets_per_block - 1) / targets_per_block);
    p.n_tiles = (int)((n_src + ts - 1) / ts);
    const int64_t want = (int64_t)WAVES * slots;
    int64_t s = (want + p.n_tblocks - 1) / p.n_tblocks;
    if (s < 1) s = 1;
    if (s > p.n_tiles) s = p.n_tiles;
    p.tiles_per_chunk = (int)((p.n_tiles + s - 1) / s);
    p.n_chunks = (p.n_tiles + p.tiles_per_chunk - 1) / p.tiles_per_chunk;
    return p;
}

// The force kernel a launch uses and its launch shape.
struct KSel {
    void* fn;
    int nt, tpb, ts;
    size_t smem;       // dynamic shared memory
    int key;           // index of its cached occupancy (0..5)
    bool mixed;
};

KSel select_kernel(int dim, int precision, double eps2) {
    KSel k;
    k.mixed = (precision == SSS_PREC_MIXED);
    if (k.mixed) {
        k.fn = (dim == 3) ? (void*)k_force_mixed<3, MIX_R, MIX_NT, MIX_TS, MIX_SUB, MIX_MINB>
                          : (void*)k_force_mixed<2, MIX_R, MIX_NT, MIX_TS, MIX_SUB, MIX_MINB>;
        k.nt = MIX_NT;
        k.tpb = MIX_NT * MIX_R;
        k.ts = MIX_TS;
        k.smem = 2 * (size_t)MIX_TS * 2 * sizeof(float4);
        k.key = 4 + (dim == 3);
        return k;
    }
    // the integer-seeded series needs r2 >= 2^-126; smaller softening takes CUDA's rsqrt
    const bool iseed = eps2 >= kIseedMinR2;
    if (iseed)
        k.fn = (dim == 3) ? (void*)k_force_f64<3, F64_R, F64_NT, F64_TS, 2, F64_MINB, F64_UNROLL>
                          : (void*)k_force_f64<2, F64_R, F64_NT, F64_TS, 2, F64_MINB, F64_UNROLL>;
    else
        k.fn = (dim == 3) ? (void*)k_force_f64<3, F64_R, F64_NT, F64_TS, 1, F64_MINB, F64_UNROLL>
                          : (void*)k_force_f64<2, F64_R, F64_NT, F64_TS, 1, F64_MINB, F64_UNROLL>;
    k.nt = F64_NT;
    k.tpb = F64_NT * F64_R;
    k.ts = F64_TS;
    k.smem = 2 * (size_t)F64_TS * sizeof(double4);
    k.key = (iseed ? 0 : 2) + (dim == 3);
    return k;
}

// Bytes of mixed-precision tile copies and tile centres for n_tiles tiles.
size_t mixed_tile_bytes(int n_tiles) { return (size_t)n_tiles * MIX_TS * 2 * sizeof(float4); }
size_t mixed_centre_bytes(int n_tiles) { return ((size_t)n_tiles * sizeof(double4) + 255) & ~(size_t)255; }

cudaError_t launch_prep(int dim, const double4* src, int64_t n_src, int n_tiles, float4* tiles,
                        double4* centres, cudaStream_t s) {
    if (dim == 3) k_prep_mixed<3, MIX_TS><<<n_tiles, 256, 0, s>>>(src, n_src, tiles, centres);
    else k_prep_mixed<2, MIX_TS><<<n_tiles, 256, 0, s>>>(src, n_src, tiles, centres);
    return cudaGetLastError();
}

// CTAs per SM of a force kernel (sets its shared-memory attribute first).
cudaError_t query_occupancy(const KSel& k, int* per_sm) {
    cudaError_t e = cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k.fn, k.nt, k.smem);
    *per_sm = n < 1 ? 1 : n;
    return e;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

int force_eval(sss_ctx* ctx, int dim, int precision, const double4* src, int64_t n_src,
               const double4* tgt, int64_t n_tgt, double eps2, const Epi& epi, cudaStream_t stream) {
    if (n_tgt <= 0) return SSS_OK;
    if (n_src <= 0) return sss_set_err(ctx, SSS_ERR_ARG, "all-pairs: n_src must be >= 1");
    if (n_src > ((int64_t)1 << 40) || n_tgt > ((int64_t)1 << 40))
        return sss_set_err(ctx, SSS_ERR_ARG, "all-pairs: size out of range");
    if (precision == SSS_PREC_MIXED_TC)
        return sss_ap::force_eval_tc(ctx, dim, src, n_src, tgt, n_tgt, eps2, epi, stream);
    const KSel ks = select_kernel(dim, precision, eps2);
    if (ctx->occ[ks.key] == 0) {
        int per_sm = 0;
        SSS_CUDA_TRY(ctx, query_occupancy(ks, &per_sm));
        ctx->occ[ks.key] = per_sm;
    }
    const Plan pl = make_plan(n_src, n_tgt, ks.tpb, ks.ts, ctx->occ[ks.key] * ctx->num_sms);

    ForceArgs a;
    memset(&a, 0, sizeof(a));
    a.src = src;
    a.n_src = n_src;
    a.tgt = tgt;
    a.n_tgt = n_tgt;
    a.eps2 = eps2;
    a.status = ctx->d_status;
    a.epi = epi;
    a.n_tiles = pl.n_tiles;
    a.n_chunks = pl.n_chunks;
    a.tiles_per_chunk = pl.tiles_per_chunk;

    // scratch: [mixed tiles][centres][partials]
    const size_t bytes_tiles = ks.mixed ? mixed_tile_bytes(pl.n_tiles) : 0;
    const size_t bytes_cent = ks.mixed ? mixed_centre_bytes(pl.n_tiles) : 0;
    const size_t bytes_part = pl.n_chunks > 1 ? (size_t)pl.n_chunks * (size_t)n_tgt * sizeof(double4) : 0;
    void* scr = nullptr;
    const size_t total = bytes_tiles + bytes_cent + bytes_part;
    if (total > 0) {
        int rc = sss_scratch(ctx, total, &scr);
        if (rc) return rc;
    }
    if (ks.mixed) {
        a.srcf = (const float4*)scr;
        a.centers = (const double4*)((char*)scr + bytes_tiles);
    }
    if (pl.n_chunks > 1) {
        a.part = (double4*)((char*)scr + bytes_tiles + bytes_cent);
        int rc = sss_counters(ctx, (size_t)pl.n_tblocks, &a.counters);
        if (rc) return rc;
    }
    if (ks.mixed) {
        cudaError_t e = launch_prep(dim, src, n_src, pl.n_tiles, (float4*)a.srcf, (double4*)a.centers, stream);
        if (e != cudaSuccess) return sss_cuda_err(ctx, e, "k_prep_mixed launch");
    }
    const unsigned grid = (unsigned)pl.n_tblocks * (unsigned)pl.n_chunks;
    void* args[] = {&a};
    SSS_CUDA_TRY(ctx, cudaLaunchKernel(ks.fn, dim3(grid), dim3(ks.nt), args, ks.smem, stream));
    return SSS_OK;
}

int check_common(sss_ctx* ctx, int dim, int precision) {
    if (!ctx) return SSS_ERR_ARG;
    if (dim != 2 && dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
    if (precision != SSS_PREC_F64 && precision != SSS_PREC_MIXED && precision != SSS_PREC_MIXED_TC)
        return sss_set_err(ctx, SSS_ERR_ARG,
                           "precision must be SSS_PREC_F64, SSS_PREC_MIXED or SSS_PREC_MIXED_TC (got %d)", precision);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    return SSS_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" int sss_allpairs_accel(sss_ctx* ctx, int dim, int precision, const double* src4, int64_t n_src,
                                  const double* tgt4, int64_t n_tgt, double* acc4, double eps2,
                                  void* stream) {
    int rc = check_common(ctx, dim, precision);
    if (rc) return rc;
    if (n_tgt < 0 || n_src < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n_tgt == 0) return SSS_OK;
    if (!src4 || !tgt4 || !acc4) return sss_set_err(ctx, SSS_ERR_ARG, "NULL pointer");
    if (!aligned16(src4) || !aligned16(tgt4) || !aligned16(acc4))
        return sss_set_err(ctx, SSS_ERR_ARG, "pointers must be 16-byte aligned");
    if (!(eps2 >= 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "eps2 must be >= 0");
    Epi e;
    memset(&e, 0, sizeof(e));
    e.mode = 0;
    e.acc = (double4*)acc4;
    return force_eval(ctx, dim, precision, (const double4*)src4, n_src, (const double4*)tgt4, n_tgt, eps2, e,
                      (cudaStream_t)stream);
}

extern "C" int sss_allpairs_potential(sss_ctx* ctx, int dim, const double* src4, int64_t n_src,
                                      const double* tgt4, int64_t n_tgt, double* phi, double eps2,
                                      void* stream) {
    int rc = check_common(ctx, dim, SSS_PREC_F64);
    if (rc) return rc;
    if (n_tgt < 0 || n_src < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative size");
    if (n_tgt == 0) return SSS_OK;
    if (!src4 || !tgt4 || !phi) return sss_set_err(ctx, SSS_ERR_ARG, "NULL pointer");
    const unsigned grid = (unsigned)((n_tgt + 255) / 256);
    if (dim == 3)
        k_potential<3><<<grid, 256, 0, (cudaStream_t)stream>>>((const double4*)src4, n_src, (const double4*)tgt4,
                                                                n_tgt, phi, eps2);
    else
        k_potential<2><<<grid, 256, 0, (cudaStream_t)stream>>>((const double4*)src4, n_src, (const double4*)tgt4,
                                                                n_tgt, phi, eps2);
    SSS_LAUNCH_CHECK(ctx, "k_potential launch");
    return SSS_OK;
}

static int check_state(sss_ctx* ctx, const sss_selfgrav_state* st) {
    if (!st) return sss_set_err(ctx, SSS_ERR_ARG, "NULL state");
    int rc = check_common(ctx, st->dim, st->precision);
    if (rc) return rc;
    if (st->n_src < 1) return sss_set_err(ctx, SSS_ERR_ARG, "state needs at least one massive body");
    if (st->n_tracer < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative tracer count");
    if (st->cur != 0 && st->cur != 1) return sss_set_err(ctx, SSS_ERR_ARG, "cur must be 0 or 1");
    if (!st->pos4[0] || !st->pos4[1] || !st->vel4 || !st->acc4) return sss_set_err(ctx, SSS_ERR_ARG, "NULL buffer");
    if (!aligned16(st->pos4[0]) || !aligned16(st->pos4[1]) || !aligned16(st->vel4) || !aligned16(st->acc4))
        return sss_set_err(ctx, SSS_ERR_ARG, "buffers must be 16-byte aligned");
    if (!(st->eps2 > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "softening must be positive");
    return SSS_OK;
}

extern "C" int sss_selfgrav_init_accel(sss_ctx* ctx, sss_selfgrav_state* st, void* stream) {
    int rc = check_state(ctx, st);
    if (rc) return rc;
    const int64_t n_all = st->n_src + st->n_tracer;
    const double4* pos = (const double4*)st->pos4[st->cur];
    Epi e;
    memset(&e, 0, sizeof(e));
    e.mode = 0;
    e.acc = (double4*)st->acc4;
    return force_eval(ctx, st->dim, st->precision, pos, st->n_src, pos, n_all, st->eps2, e, (cudaStream_t)stream);
}

extern "C" int sss_selfgrav_step_batch(sss_ctx* ctx, sss_selfgrav_state* st, int integrator, double dt,
                                       int steps, float* snap, void* stream) {
    int rc = check_state(ctx, st);
    if (rc) return rc;
    if (steps < 1) return sss_set_err(ctx, SSS_ERR_ARG, "steps must be >= 1 (got %d)", steps);
    if (integrator != SSS_INT_KDK && integrator != SSS_INT_YOSHIDA4)
        return sss_set_err(ctx, SSS_ERR_ARG, "unknown integrator %d", integrator);
    if (!(dt == dt)) return sss_set_err(ctx, SSS_ERR_ARG, "dt is NaN");
    cudaStream_t s = (cudaStream_t)stream;
    const int D = st->dim;
    const int64_t n_all = st->n_src + st->n_tracer;
    const int64_t row = 2 * (int64_t)D * st->n_src + (int64_t)D * st->n_tracer;

    // substep weights (Yoshida 1990 fourth-order triple-jump composition)
    double w[3];
    int nsub;
    if (integrator == SSS_INT_KDK) {
        nsub = 1;
        w[0] = 1.0;
    } else {
        const double cbrt2 = cbrt(2.0);
        nsub = 3;
        w[0] = 1.0 / (2.0 - cbrt2);
        w[1] = -cbrt2 / (2.0 - cbrt2);
        w[2] = w[0];
    }

    // opening half kick + drift of the first substep
    {
        const double4* p = (const double4*)st->pos4[st->cur];
        double4* q = (double4*)st->pos4[1 - st->cur];
        const unsigned grid = (unsigned)((n_all + 255) / 256);
        if (D == 3)
            k_open<3><<<grid, 256, 0, s>>>(p, q, (double4*)st->vel4, (const double4*)st->acc4, n_all,
                                          0.5 * w[0] * dt, w[0] * dt);
        else
            k_open<2><<<grid, 256, 0, s>>>(p, q, (double4*)st->vel4, (const double4*)st->acc4, n_all,
                                          0.5 * w[0] * dt, w[0] * dt);
        SSS_LAUNCH_CHECK(ctx, "k_open launch");
        st->cur = 1 - st->cur;
    }
    for (int step = 0; step < steps; ++step) {
        for (int k = 0; k < nsub; ++k) {
            Epi e;
            memset(&e, 0, sizeof(e));
            e.mode = 1;
            e.last = (step == steps - 1 && k == nsub - 1) ? 1 : 0;
            e.acc = (double4*)st->acc4;
            e.vel = (double4*)st->vel4;
            e.pos_nxt = (double4*)st->pos4[1 - st->cur];
            e.snap = (snap && k == nsub - 1) ? snap + (int64_t)step * row : nullptr;
            e.kc = 0.5 * w[k] * dt;
            const int kn = (k + 1) % nsub;
            e.ko = 0.5 * w[kn] * dt;
            e.kd = w[kn] * dt;
            e.n_src = st->n_src;
            e.n_tr = st->n_tracer;
            const double4* pos = (const double4*)st->pos4[st->cur];
            rc = force_eval(ctx, D, st->precision, pos, st->n_src, pos, n_all, st->eps2, e, s);
            if (rc) return rc;
            st->cur = 1 - st->cur;
        }
    }
    return SSS_OK;
}

// ------------------------------------------------ no-allocation variant
//
// sss_allpairs_accel_noalloc: the all-pairs force of sss_allpairs_accel for
// callers that must not allocate device memory (see include/sss.h). Its
// scratch (status word, chunk-arrival counters, mixed-precision tiles and
// chunk partial sums) lives in the file-scope array below, which every GPU
// that loads libsss holds until the process exits. Host code reaches the
// array only through the device address cudaGetSymbolAddress returns; the
// symbol itself names a host-side stand-in.

#define SSS_NOALLOC_STATUS_BYTES 256u
#define SSS_NOALLOC_COUNTERS 16384u

static __device__ __align__(256) unsigned char g_sss_noalloc_scratch[SSS_NOALLOC_SCRATCH_BYTES];

// The stated mixed-precision source limit must be exactly what the scratch
// layout holds: whole tiles plus their 256-byte-rounded centres.
constexpr size_t noalloc_fixed_bytes(size_t n_src) {
    return ((n_src + MIX_TS - 1) / MIX_TS) * MIX_TS * 2 * sizeof(float4) +
           ((((n_src + MIX_TS - 1) / MIX_TS) * sizeof(double4) + 255) & ~(size_t)255);
}
constexpr size_t kNoAllocAvail =
    (size_t)SSS_NOALLOC_SCRATCH_BYTES - SSS_NOALLOC_STATUS_BYTES - SSS_NOALLOC_COUNTERS * sizeof(unsigned);
static_assert(noalloc_fixed_bytes(SSS_NOALLOC_MAX_MIXED_SOURCES) <= kNoAllocAvail &&
                  noalloc_fixed_bytes(SSS_NOALLOC_MAX_MIXED_SOURCES + 1) > kNoAllocAvail,
              "SSS_NOALLOC_MAX_MIXED_SOURCES does not match the no-allocation scratch layout");

namespace {

struct NoAllocDevice {
    int ready;
    unsigned char* base;  // device address of g_sss_noalloc_scratch on this device
    int num_sms;
    int occ[6];           // CTAs per SM of the force kernels (KSel::key)
};

constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
pthread_mutex_t g_noalloc_mu = PTHREAD_MUTEX_INITIALIZER;

int noalloc_err(char* buf, size_t len, int code, const char* fmt, ...) {
    if (buf && len) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, len, fmt, ap);
        va_end(ap);
    }
    return code;
}

// Once per device, with that device current: resolve the scratch array's
// device address and the launch parameters of the force kernels.
int noalloc_setup(int device, NoAllocDevice** out, char* eb, size_t el) {
    pthread_mutex_lock(&g_noalloc_mu);
    NoAllocDevice* d = &g_noalloc_dev[device];
    int rc = SSS_OK;
    if (!d->ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sss_noalloc_scratch);
        if (e != cudaSuccess) {
            rc = noalloc_err(eb, el, SSS_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        } else if (((uintptr_t)p & 255u) != 0) {
            rc = noalloc_err(eb, el, SSS_ERR_CUDA, "static scratch is not 256-byte aligned");
        } else {
            d->base = (unsigned char*)p;
            e = cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, device);
            // one representative eps2 per f64 seed variant selects each kernel once
            const double probe_eps2[2] = {1.0, 0.0};
            for (int prec = 0; prec < 2 && e == cudaSuccess; ++prec)
                for (int dim = 2; dim <= 3 && e == cudaSuccess; ++dim)
                    for (int v = 0; v < (prec ? 1 : 2) && e == cudaSuccess; ++v) {
                        const KSel ks = select_kernel(dim, prec, probe_eps2[v]);
                        e = query_occupancy(ks, &d->occ[ks.key]);
                    }
            if (e != cudaSuccess)
                rc = noalloc_err(eb, el, SSS_ERR_CUDA, "no-alloc setup: %s", cudaGetErrorString(e));
            else
                d->ready = 1;
        }
    }
    pthread_mutex_unlock(&g_noalloc_mu);
    *out = d;
    return rc;
}

}  // namespace

extern "C" int sss_allpairs_accel_noalloc(int device, int dim, int precision, const double* src4, int64_t n_src,
                                          const double* tgt4, int64_t n_tgt, double* acc4, double eps2,
                                          int* d_status, void* stream, char* errbuf, size_t errbuf_len) {
    char* eb = errbuf;
    const size_t el = errbuf_len;
    if (dim != 2 && dim != 3) return noalloc_err(eb, el, SSS_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
    if (precision != SSS_PREC_F64 && precision != SSS_PREC_MIXED)
        return noalloc_err(eb, el, SSS_ERR_ARG, "unknown precision %d", precision);
    if (n_src < 0 || n_tgt < 0) return noalloc_err(eb, el, SSS_ERR_ARG, "negative size");
    if (n_tgt == 0) return SSS_OK;
    if (n_src < 1) return noalloc_err(eb, el, SSS_ERR_ARG, "n_src must be >= 1");
    if (n_src > ((int64_t)1 << 40) || n_tgt > ((int64_t)1 << 40))
        return noalloc_err(eb, el, SSS_ERR_ARG, "size out of range");
    if (!src4 || !tgt4 || !acc4) return noalloc_err(eb, el, SSS_ERR_ARG, "NULL pointer");
    if (!aligned16(src4) || !aligned16(tgt4) || !aligned16(acc4) || ((uintptr_t)d_status & 3u))
        return noalloc_err(eb, el, SSS_ERR_ARG, "pointers must be 16-byte aligned (status 4-byte)");
    if (!(eps2 >= 0.0)) return noalloc_err(eb, el, SSS_ERR_ARG, "eps2 must be >= 0");
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev || device >= kNoAllocMaxDevices)
        return noalloc_err(eb, el, SSS_ERR_ARG, "bad device %d", device);
    if (cudaSetDevice(device) != cudaSuccess) return noalloc_err(eb, el, SSS_ERR_CUDA, "cudaSetDevice failed");
    NoAllocDevice* d = nullptr;
    int rc = noalloc_setup(device, &d, eb, el);
    if (rc) return rc;

    const KSel ks = select_kernel(dim, precision, eps2);
    Plan pl = make_plan(n_src, n_tgt, ks.tpb, ks.ts, d->occ[ks.key] * d->num_sms);

    // scratch layout: [status 256 B][counters 64 KiB][tiles][centres][partials]
    const size_t data_off = SSS_NOALLOC_STATUS_BYTES + SSS_NOALLOC_COUNTERS * sizeof(unsigned);
    const size_t avail = (size_t)SSS_NOALLOC_SCRATCH_BYTES - data_off;
    const size_t bytes_tiles = ks.mixed ? mixed_tile_bytes(pl.n_tiles) : 0;
    const size_t bytes_cent = ks.mixed ? mixed_centre_bytes(pl.n_tiles) : 0;
    const size_t fixed = bytes_tiles + bytes_cent;
    if (fixed > avail)
        return noalloc_err(eb, el, SSS_ERR_CAPACITY,
                           "n_src = %lld needs %zu bytes of mixed-precision tiles; the no-allocation "
                           "scratch holds %zu (at most %d sources)", (long long)n_src, fixed, avail,
                           SSS_NOALLOC_MAX_MIXED_SOURCES);
    // narrow the source split until its partial sums fit (1 chunk needs none)
    if (pl.n_chunks > 1) {
        const size_t per_chunk = (size_t)n_tgt * sizeof(double4);
        size_t s_fit = (avail - fixed) / per_chunk;
        if (pl.n_tblocks > (int)SSS_NOALLOC_COUNTERS) s_fit = 1;
        if (s_fit < (size_t)pl.n_chunks) {
            if (s_fit <= 1) {
                pl.tiles_per_chunk = pl.n_tiles;
                pl.n_chunks = 1;
            } else {
                pl.tiles_per_chunk = (int)((pl.n_tiles + s_fit - 1) / s_fit);
                pl.n_chunks = (pl.n_tiles + pl.tiles_per_chunk - 1) / pl.tiles_per_chunk;
            }
        }
    }
    unsigned char* base = d->base;
    cudaStream_t s = (cudaStream_t)stream;
    int* status = d_status ? d_status : (int*)base;
    unsigned* counters = (unsigned*)(base + SSS_NOALLOC_STATUS_BYTES);
    unsigned char* data = base + data_off;

    ForceArgs a;
    memset(&a, 0, sizeof(a));
    a.src = (const double4*)src4;
    a.n_src = n_src;
    a.tgt = (const double4*)tgt4;
    a.n_tgt = n_tgt;
    a.eps2 = eps2;
    a.n_tiles = pl.n_tiles;
    a.n_chunks = pl.n_chunks;
    a.tiles_per_chunk = pl.tiles_per_chunk;
    a.status = status;
    a.epi.mode = 0;
    a.epi.acc = (double4*)acc4;
    if (ks.mixed) {
        a.srcf = (const float4*)data;
        a.centers = (const double4*)(data + bytes_tiles);
    }
    if (pl.n_chunks > 1) {
        a.part = (double4*)(data + fixed);
        a.counters = counters;
    }

    // the array keeps the previous call's contents: zero what must start at 0
    cudaError_t e = cudaSuccess;
    if (!d_status) e = cudaMemsetAsync(status, 0, sizeof(int), s);
    if (e == cudaSuccess && pl.n_chunks > 1)
        e = cudaMemsetAsync(counters, 0, (size_t)pl.n_tblocks * sizeof(unsigned), s);
    if (e != cudaSuccess) return noalloc_err(eb, el, SSS_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    if (ks.mixed) {
        e = launch_prep(dim, a.src, n_src, pl.n_tiles, (float4*)a.srcf, (double4*)a.centers, s);
        if (e != cudaSuccess) return noalloc_err(eb, el, SSS_ERR_CUDA, "k_prep_mixed: %s", cudaGetErrorString(e));
    }
    const unsigned grid = (unsigned)pl.n_tblocks * (unsigned)pl.n_chunks;
    void* args[] = {&a};
    e = cudaLaunchKernel(ks.fn, dim3(grid), dim3(ks.nt), args, ks.smem, s);
    if (e != cudaSuccess) return noalloc_err(eb, el, SSS_ERR_CUDA, "force kernel: %s", cudaGetErrorString(e));
    return SSS_OK;
}
