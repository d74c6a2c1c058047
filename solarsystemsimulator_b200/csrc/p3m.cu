// Short-range part of a P3M force in the periodic box, for the 3-D particle
// mesh (pm3d.cu). The mesh's Green's function -4 pi G / k^2 e^{-k^2 r_s^2} is
// the force of Gaussian clouds; what it leaves out of a pair at distance r
// is G m g(alpha r) / r^2 along the separation, alpha = 1 / (2 r_s) and
// g(x) = erfc(x) + 2 x e^{-x^2} / sqrt(pi): the real-space term of an Ewald
// sum with that alpha. With the Plummer softening of the direct sum the pair
// adds ((1 + eps^2 / r^2)^{-3/2} - 1) / r^2 as well. Both act for r < r_cut
// (g(alpha r_cut) is the truncation error of a pair at the cutoff, relative to
// its Newtonian term: 4.4e-4 for alpha r_cut = 3, 2e-5 for 3.5).
// The reference has no such term: its 2-D PM (pm_kernel.py:63-154) ends at
// the mesh force; here it is the exact short-range part of the force the
// learned correction then refines.
//
//   keys    : chaining cell (side box / M >= r_cut) of every particle
//   sort    : stable radix sort by cell (devscan.cuh), particles gathered in
//             that order as (x, y, z, m)
//   bounds  : first and last sorted particle of every cell
//   items   : one work item per group of 32 particles of a cell (cells
//             hold from none to many thousands in a clustered state)
//   pairs   : persistent warps take items from a counter (a dense cell's
//             items spread over many warps). Every pair is evaluated once
//             (the two accelerations are m_j h d and -m_i h d): an item pairs
//             its particles with each other, with the later particles of its
//             cell and with the particles of the neighbouring cells of
//             higher index (13 or so of the 26, periodic). The sources are
//             staged through the warp's shared memory in chunks of 32,
//             relative to the item's cell corner, so that f32 differences
//             keep the positions' resolution; lane l meets sources (l + k)
//             and (l + k + 16) mod 32 at step k, in packed f32x2 arithmetic,
//             and the sources' sums rotate through the lanes with them, so
//             that both sides accumulate in registers. Both go to an f32
//             accumulator per particle with atomics.
//   finish  : acceleration = mesh force (already in a) + G x accumulator, in
//             f64, through the KDK epilogue of the force passes.

#include "pm3d.cuh"
#include "devscan.cuh"

namespace {

constexpr int PP_WARPS = 4;                         // cells per block

unsigned blocks_for(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

__global__ void k_pp_keys(const Pm3Parts s, int M, double inv_l, unsigned long long* __restrict__ keys,
                          unsigned* __restrict__ vals) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    int c[3];
    for (int d = 0; d < 3; ++d) {
        const double f = s.x[d][p] * inv_l;
        const int ci = f >= 0.0 ? (int)f : 0;              // NaN and negatives go to cell 0
        c[d] = min(ci, M - 1);
    }
    keys[p] = ((unsigned long long)c[2] * M + c[1]) * M + c[0];
    vals[p] = (unsigned)p;
}

__global__ void k_pp_gather(const Pm3Parts s, const unsigned* __restrict__ order, double4* __restrict__ src) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= s.n) return;
    const unsigned p = order[q];
    src[q] = make_double4(s.x[0][p], s.x[1][p], s.x[2][p], s.m ? s.m[p] : s.mass_const);
}

// first and one-past-last sorted position of every occupied cell (the
// others stay 0, 0)
__global__ void k_pp_bounds(const unsigned long long* __restrict__ keys, long long n, int* __restrict__ first,
                            int* __restrict__ last) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const unsigned long long k = keys[q];
    if (q == 0 || keys[q - 1] != k) first[k] = (int)q;
    if (q == n - 1 || keys[q + 1] != k) last[k] = (int)(q + 1);
}

// items of each cell: ceil(count / 32)
__global__ void k_pp_groups(const int* __restrict__ first, const int* __restrict__ last, long long cells,
                            long long* __restrict__ groups) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < cells) groups[c] = (last[c] - first[c] + 31) / 32;
}

// item list: (cell, first target) of every group, in cell order; the
// number of items into *n_items
__global__ void k_pp_items(const int* __restrict__ first, const long long* __restrict__ offs, long long cells,
                           const long long* __restrict__ groups, int2* __restrict__ items,
                           unsigned* __restrict__ n_items) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    const long long g = groups[c], o = offs[c];
    for (long long k = 0; k < g; ++k) items[o + k] = make_int2((int)c, first[c] + 32 * (int)k);
    if (c == cells - 1) *n_items = (unsigned)(o + g);
}

struct PPArgs {
    const double4* src;             // particles in cell order: x, y, z, m
    const unsigned* order;          // cell order -> particle index
    const int* first;               // M^3
    const int* last;
    int M;
    double l;                       // chaining cell side
    double box;
    double G;
    float alpha, rc2, eps2;
    const int2* items;
    const unsigned* n_items;
    unsigned* next;                 // work counter (zero at launch)
    float* acc;                     // 3 x n, by cell-order position (zero at launch)
    long long n;
};

// ---- packed f32x2 pair arithmetic: two sources per lane and step
typedef unsigned long long f2x;                     // two packed f32

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
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ f2x shfl2(f2x v, int from) {
    return __shfl_sync(0xffffffffu, v, from);
}

// h(r) of a pair (a_i += m_j h d, a_j -= m_i h d, d = x_j - x_i), for
// 0 < r < r_cut: (g(x) + (1 + u)^{-3/2} - 1) / r^3 with u = eps^2 / r^2,
// evaluated as (g - 1) / r^3 + (r^2 + eps^2)^{-3/2} (its rounding is about
// 1e-7 of the pair's Newtonian term 1 / r^2 for every r). erfc(x) =
// e^{-x^2} t (a1 + a2 t + ... + a5 t^4), t = 1 / (1 + p x) (Abramowitz &
// Stegun 7.1.26, |error| <= 1.5e-7), so g shares its Gaussian with the
// second term 2 x e^{-x^2} / sqrt(pi). No branches: out of range (and for
// coincident particles, where the arithmetic is not finite) the caller
// selects 0. Two pairs at a time in packed f32x2 arithmetic; the reciprocal
// square roots, the exponential and the reciprocal are f32 MUFU operations.
__device__ __forceinline__ f2x pp_h2(f2x R2, const f2x* K) {
    // K: alpha, -log2(e), p, 1, a1..a5, 2/sqrt(pi), eps^2, -1 (each in both halves)
    float r0, r1;
    upk2(R2, r0, r1);
    const f2x RI = pk2(sss_rsqrt_approx_f32(r0), sss_rsqrt_approx_f32(r1));
    const f2x INV3 = mul2(mul2(RI, RI), RI);
    const f2x X = mul2(K[0], mul2(R2, RI));
    float v0, v1;
    upk2(mul2(mul2(X, X), K[1]), v0, v1);
    const f2x EX = pk2(ex2_approx(v0), ex2_approx(v1));
    float d0, d1;
    upk2(fma2(K[2], X, K[3]), d0, d1);
    const f2x T = pk2(rcp_approx(d0), rcp_approx(d1));
    const f2x POLY = mul2(T, fma2(T, fma2(T, fma2(T, fma2(T, K[8], K[7]), K[6]), K[5]), K[4]));
    const f2x G = mul2(EX, fma2(K[9], X, POLY));
    float s0, s1;
    upk2(add2(R2, K[10]), s0, s1);
    const f2x SI = pk2(sss_rsqrt_approx_f32(s0), sss_rsqrt_approx_f32(s1));
    return fma2(add2(G, K[11]), INV3, mul2(mul2(SI, SI), SI));
}

// One chunk of sources against the lanes' targets, two sources per step:
// offsets (a, a + da) for steps a = a0 .. a1 - 1 (source (lane + offset) mod
// 32); `own` masks offset 16 on lanes 16 .. 31 (the item's own chunk, whose
// pairs (l, l + 16) and (l + 16, l) coincide). Both sources' sums rotate
// through the lanes and end on their own lanes, then go to the accumulator.
__device__ __forceinline__ void pp_chunk2(const float4* stage, int lane, int a0, int a1, int da, bool own,
                                          f2x NTX, f2x NTY, f2x NTZ, f2x NTM, const f2x* K,
                                          const PPArgs& q, f2x& AX, f2x& AY, f2x& AZ, long long src0, int m) {
    f2x BX = 0ull, BY = 0ull, BZ = 0ull;             // sums of sources (lane + a) and (lane + a + da)
#pragma unroll 2
    for (int a = a0; a < a1; ++a) {
        const float4 sa = stage[(lane + a) & 31], sb = stage[(lane + a + da) & 31];
        const f2x DX = add2(pk2(sa.x, sb.x), NTX), DY = add2(pk2(sa.y, sb.y), NTY), DZ = add2(pk2(sa.z, sb.z), NTZ);
        const f2x R2 = fma2(DX, DX, fma2(DY, DY, mul2(DZ, DZ)));
        float r0, r1;
        upk2(R2, r0, r1);
        const bool in0 = r0 < q.rc2 && r0 > 0.0f;
        const bool in1 = r1 < q.rc2 && r1 > 0.0f && !(own && a + da == 16 && lane >= 16);
        if (__any_sync(0xffffffffu, in0 || in1)) {                  // (warp-uniform)
            float h0, h1;
            upk2(pp_h2(R2, K), h0, h1);
            const f2x H = pk2(in0 ? h0 : 0.0f, in1 ? h1 : 0.0f);
            const f2x HJ = mul2(H, pk2(sa.w, sb.w)), HI = mul2(H, NTM);
            AX = fma2(HJ, DX, AX);
            AY = fma2(HJ, DY, AY);
            AZ = fma2(HJ, DZ, AZ);
            BX = fma2(HI, DX, BX);
            BY = fma2(HI, DY, BY);
            BZ = fma2(HI, DZ, BZ);
        }
        if (a + 1 < a1) {                                          // take the next lane's sums (sources + 1)
            const int from = (lane + 1) & 31;
            BX = shfl2(BX, from);
            BY = shfl2(BY, from);
            BZ = shfl2(BZ, from);
        }
    }
    // lane l holds sources (l + a1 - 1) and (l + a1 - 1 + da): deliver both to their lanes
    const int fa = (lane - (a1 - 1)) & 31, fb = (lane - (a1 - 1 + da)) & 31;
    float xa, xb, ya, yb, za, zb, t0, t1;
    upk2(shfl2(BX, fa), xa, t0);
    upk2(shfl2(BX, fb), t1, xb);
    upk2(shfl2(BY, fa), ya, t0);
    upk2(shfl2(BY, fb), t1, yb);
    upk2(shfl2(BZ, fa), za, t0);
    upk2(shfl2(BZ, fb), t1, zb);
    if (lane < m) {
        atomicAdd(q.acc + src0 + lane, xa + xb);
        atomicAdd(q.acc + q.n + src0 + lane, ya + yb);
        atomicAdd(q.acc + 2 * q.n + src0 + lane, za + zb);
    }
}

__global__ void __launch_bounds__(PP_WARPS * 32) k_pp_pairs(const PPArgs q) {
    __shared__ float4 sh[PP_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int M = q.M;
    const unsigned total = *q.n_items;
    float4* stage = sh[w];
    const f2x K[12] = {pk2(q.alpha, q.alpha), pk2(-1.44269504f, -1.44269504f), pk2(0.3275911f, 0.3275911f),
                       pk2(1.0f, 1.0f), pk2(0.254829592f, 0.254829592f), pk2(-0.284496736f, -0.284496736f),
                       pk2(1.421413741f, 1.421413741f), pk2(-1.453152027f, -1.453152027f),
                       pk2(1.061405429f, 1.061405429f), pk2(1.12837917f, 1.12837917f), pk2(q.eps2, q.eps2),
                       pk2(-1.0f, -1.0f)};
    for (;;) {
        unsigned it = 0;
        if (lane == 0) it = atomicAdd(q.next, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= total) break;
        const int2 item = q.items[it];
        const int c = item.x, t0 = item.y, cl = q.last[c];
        const int t = t0 + lane;
        const bool act = t < cl;
        const int cx = c % M, cy = (c / M) % M, cz = c / (M * M);
        const double ox = cx * q.l, oy = cy * q.l, oz = cz * q.l;
        float tx = 0.0f, ty = 0.0f, tz = 0.0f, tm = 0.0f;
        if (act) {
            const double4 p = q.src[t];
            tx = (float)(p.x - ox);
            ty = (float)(p.y - oy);
            tz = (float)(p.z - oz);
            tm = (float)p.w;
        }
        const f2x NTX = pk2(-tx, -tx), NTY = pk2(-ty, -ty), NTZ = pk2(-tz, -tz), NTM = pk2(-tm, -tm);
        f2x AX = 0ull, AY = 0ull, AZ = 0ull;
        // the item's own particles with each other (offsets 1 .. 16 as (j, j + 8), j = 1 .. 8)
        __syncwarp();
        stage[lane] = make_float4(tx, ty, tz, tm);
        __syncwarp();
        pp_chunk2(stage, lane, 1, 9, 8, true, NTX, NTY, NTZ, NTM, K, q, AX, AY, AZ, t0, min(32, cl - t0));
        // the later particles of the cell, then the neighbouring cells of higher index
        for (int nb = -1; nb < 27; ++nb) {
            int s0, s1;
            double sx = -ox, sy = -oy, sz = -oz;                    // source shift: periodic image - corner
            if (nb < 0) {
                s0 = t0 + 32;
                s1 = cl;
            } else {
                if (nb == 13) continue;                            // the cell itself
                int nx = cx + nb % 3 - 1, ny = cy + (nb / 3) % 3 - 1, nz = cz + nb / 9 - 1;
                if (nx < 0) { nx += M; sx -= q.box; } else if (nx >= M) { nx -= M; sx += q.box; }
                if (ny < 0) { ny += M; sy -= q.box; } else if (ny >= M) { ny -= M; sy += q.box; }
                if (nz < 0) { nz += M; sz -= q.box; } else if (nz >= M) { nz -= M; sz += q.box; }
                const int nc = (nz * M + ny) * M + nx;
                if (nc < c) continue;                              // that cell's items take these pairs
                s0 = q.first[nc];
                s1 = q.last[nc];
            }
            for (int j0 = s0; j0 < s1; j0 += 32) {
                const int j = j0 + lane;
                __syncwarp();                                      // the previous chunk is consumed
                float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (j < s1) {
                    const double4 p = q.src[j];
                    v = make_float4((float)(p.x + sx), (float)(p.y + sy), (float)(p.z + sz), (float)p.w);
                }
                stage[lane] = v;
                __syncwarp();
                pp_chunk2(stage, lane, 0, 16, 16, false, NTX, NTY, NTZ, NTM, K, q, AX, AY, AZ, j0, min(32, s1 - j0));
            }
        }
        if (act) {
            float x0, x1, y0, y1, z0, z1;
            upk2(AX, x0, x1);
            upk2(AY, y0, y1);
            upk2(AZ, z0, z1);
            atomicAdd(q.acc + t, x0 + x1);
            atomicAdd(q.acc + q.n + t, y0 + y1);
            atomicAdd(q.acc + 2 * q.n + t, z0 + z1);
        }
    }
}

// acceleration = mesh force + G x pair sums, then the epilogue
__global__ void k_pp_finish(const PPArgs q, const Pm3Parts s, const Pm3Epi e) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= s.n) return;
    const unsigned i = q.order[t];
    const long long n = q.n;
    pm3_epilogue(s, e, i, s.a[0][i] + q.G * (double)q.acc[t], s.a[1][i] + q.G * (double)q.acc[n + t],
                 s.a[2][i] + q.G * (double)q.acc[2 * n + t]);
}

}  // namespace

extern "C" int sss_pm3_short(sss_pm3* p, const sss_pm3_particles* s, double G, double alpha, double r_cut,
                             double eps, int mode, double hdt, double dt, float* snap, void* stream) {
    if (!p) return SSS_ERR_ARG;
    sss_ctx* ctx = p->ctx;
    if (!s) return sss_set_err(ctx, SSS_ERR_ARG, "NULL particle state");
    if (s->n < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative particle count");
    if (mode < SSS_PM3_FORCE || mode > SSS_PM3_KICK_DRIFT) return sss_set_err(ctx, SSS_ERR_ARG, "bad mode");
    if (!(alpha > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "alpha must be > 0");
    if (!(r_cut > 0.0) || !(eps >= 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "r_cut must be > 0, eps >= 0");
    const double mf = floor(p->box / r_cut);
    if (!(mf >= 3.0)) return sss_set_err(ctx, SSS_ERR_ARG, "r_cut must be <= box / 3");
    const int M = (int)std::min(mf, 1024.0);
    if (s->n == 0) return SSS_OK;
    if (s->n >= ((int64_t)1 << 31)) return sss_set_err(ctx, SSS_ERR_ARG, "too many particles");
    for (int c = 0; c < 3; ++c)
        if (!s->x[c] || !s->v[c] || !s->a[c]) return sss_set_err(ctx, SSS_ERR_ARG, "NULL particle array");
    SSS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const long long n = s->n;
    const long long cells = (long long)M * M * M;
    int bits = 0;
    while ((1LL << bits) < cells) ++bits;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) & ~(size_t)255; return o; };
    const size_t o_k0 = take(8 * n), o_k1 = take(8 * n), o_v0 = take(4 * n), o_v1 = take(4 * n);
    const size_t o_src = take(32 * n), o_first = take(4 * cells), o_last = take(4 * cells);
    const size_t o_rs = take(8 * std::max(sss_dev::radix_scratch(n), sss_dev::scan_scratch(cells)));
    const size_t o_grp = take(8 * cells), o_off = take(8 * cells);
    const size_t o_items = take(8 * (size_t)(n / 32 + cells + 1)), o_cnt = take(8), o_acc = take(12 * n);
    void* scr = nullptr;
    int rc = sss_scratch(ctx, off, &scr);
    if (rc) return rc;
    char* B = (char*)scr;
    unsigned long long* k0 = (unsigned long long*)(B + o_k0);
    unsigned long long* k1 = (unsigned long long*)(B + o_k1);
    unsigned* v0 = (unsigned*)(B + o_v0);
    unsigned* v1 = (unsigned*)(B + o_v1);
    double4* src = (double4*)(B + o_src);
    int* first = (int*)(B + o_first);
    int* last = (int*)(B + o_last);
    long long* groups = (long long*)(B + o_grp);
    long long* offs = (long long*)(B + o_off);
    int2* items = (int2*)(B + o_items);
    unsigned* counters = (unsigned*)(B + o_cnt);                  // [0] items, [1] work counter
    const Pm3Parts parts = pm3_parts(s);
    const double l = p->box / M;
    k_pp_keys<<<blocks_for(n, 256), 256, 0, st>>>(parts, M, 1.0 / l, k0, v0);
    SSS_LAUNCH_CHECK(ctx, "k_pp_keys");
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(k0, v0, k1, v1, n, (long long*)(B + o_rs), st, ctx->d_status, bits));
    k_pp_gather<<<blocks_for(n, 256), 256, 0, st>>>(parts, v0, src);
    SSS_LAUNCH_CHECK(ctx, "k_pp_gather");
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(first, 0, 4 * (size_t)cells, st));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(last, 0, 4 * (size_t)cells, st));
    k_pp_bounds<<<blocks_for(n, 256), 256, 0, st>>>(k0, n, first, last);
    SSS_LAUNCH_CHECK(ctx, "k_pp_bounds");
    k_pp_groups<<<blocks_for(cells, 256), 256, 0, st>>>(first, last, cells, groups);
    SSS_LAUNCH_CHECK(ctx, "k_pp_groups");
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(groups, offs, cells, (long long*)(B + o_rs), st, ctx->d_status));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(counters, 0, 8, st));
    k_pp_items<<<blocks_for(cells, 256), 256, 0, st>>>(first, offs, cells, groups, items, counters);
    SSS_LAUNCH_CHECK(ctx, "k_pp_items");
    PPArgs q;
    q.src = src;
    q.order = v0;
    q.first = first;
    q.last = last;
    q.M = M;
    q.l = l;
    q.box = p->box;
    q.G = G;
    q.alpha = (float)alpha;
    q.rc2 = (float)(r_cut * r_cut);
    q.eps2 = (float)(eps * eps);
    q.items = items;
    q.n_items = counters;
    q.next = counters + 1;
    q.acc = (float*)(B + o_acc);
    q.n = n;
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(q.acc, 0, 12 * (size_t)n, st));
    int per_sm = 0;
    SSS_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pp_pairs, PP_WARPS * 32, 0));
    const unsigned grid = (unsigned)(ctx->num_sms * std::max(per_sm, 1));
    k_pp_pairs<<<grid, PP_WARPS * 32, 0, st>>>(q);
    SSS_LAUNCH_CHECK(ctx, "k_pp_pairs");
    Pm3Epi e{mode, hdt, dt, p->box, snap};
    k_pp_finish<<<blocks_for(n, 256), 256, 0, st>>>(q, parts, e);
    SSS_LAUNCH_CHECK(ctx, "k_pp_finish");
    return SSS_OK;
}
