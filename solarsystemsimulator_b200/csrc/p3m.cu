// Short-range part of a P3M force in the periodic box, for the 3-D particle
// mesh (pm3d.cu). The mesh's Green's function -4 pi G / k^2 e^{-k^2 r_s^2} is
// the force of Gaussian clouds; what it leaves out of a pair at distance r
// is G m g(alpha r) / r^2 along the separation, alpha = 1 / (2 r_s) and
// g(x) = erfc(x) + 2 x e^{-x^2} / sqrt(pi): the real-space term of an Ewald
// sum with that alpha. With the Plummer softening of the direct sum the pair
// adds ((1 + eps^2 / r^2)^{-3/2} - 1) / r^2 as well. Both act for r < r_cut
// (g(alpha r_cut) is the truncation error; alpha r_cut = 3.5 gives 2e-5).
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
//             keep the positions' resolution; lane l meets source (l + k)
//             mod 32 at step k and the sources' sums rotate through the lanes
//             with them, so that both sides accumulate in registers. Both go
//             to an f32 accumulator per particle with atomics.
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

// h(r) of a pair (a_i += m_j h d, a_j -= m_i h d, d = x_j - x_i), for
// 0 < r < r_cut: (g(x) + (1 + u)^{-3/2} - 1) / r^3 with u = eps^2 / r^2,
// evaluated as (g - 1) / r^3 + (r^2 + eps^2)^{-3/2} (its rounding is about
// 1e-7 of the pair's Newtonian term 1 / r^2 for every r). erfc(x) =
// e^{-x^2} t (a1 + a2 t + ... + a5 t^4), t = 1 / (1 + p x) (Abramowitz &
// Stegun 7.1.26, |error| <= 1.5e-7), so g shares its Gaussian with the
// second term 2 x e^{-x^2} / sqrt(pi). No branches: out of range (and for
// coincident particles, where the arithmetic is not finite) the caller
// selects 0.
__device__ __forceinline__ float pp_h(float r2, float alpha, float eps2) {
    const float rinv = rsqrtf(r2);
    const float inv_r3 = rinv * rinv * rinv;
    const float x = alpha * (r2 * rinv);
    const float ex = __expf(-x * x);
    const float t = __fdividef(1.0f, fmaf(0.3275911f, x, 1.0f));
    const float poly =
        t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f))));
    const float g = ex * fmaf(1.12837917f, x, poly);
    const float si = rsqrtf(r2 + eps2);
    return fmaf(g - 1.0f, inv_r3, si * si * si);
}

// One chunk of sources (stage[0 .. 32), masses in w; invalid entries have
// w = 0 and the lanes without a target tm = 0) against the lanes' targets,
// steps k0 .. k1 - 1 (lane l meets source (l + k) mod 32); `half` limits
// step 16 to lanes 0 .. 15 (the item's own chunk, whose pairs (l, l + 16)
// and (l + 16, l) coincide). The sources' sums end on their own lanes and go
// to the accumulator (positions src0 .. src0 + m - 1).
__device__ __forceinline__ void pp_chunk(const float4* stage, int lane, int k0, int k1, bool half, float tx,
                                         float ty, float tz, float tm, const PPArgs& q, float& ax, float& ay,
                                         float& az, long long src0, int m) {
    float bx = 0.0f, by = 0.0f, bz = 0.0f;                         // the sum of source (lane + k) mod 32
#pragma unroll 2
    for (int k = k0; k < k1; ++k) {
        const float4 sj = stage[(lane + k) & 31];
        const float dx = sj.x - tx, dy = sj.y - ty, dz = sj.z - tz;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const bool in = r2 < q.rc2 && r2 > 0.0f && !(half && k == 16 && lane >= 16);
        if (__any_sync(0xffffffffu, in)) {                          // (warp-uniform: no divergent pair arithmetic)
            const float h0 = pp_h(r2, q.alpha, q.eps2);
            const float h = in ? h0 : 0.0f;
            const float hj = h * sj.w, hi = h * tm;
            ax = fmaf(hj, dx, ax);
            ay = fmaf(hj, dy, ay);
            az = fmaf(hj, dz, az);
            bx = fmaf(-hi, dx, bx);
            by = fmaf(-hi, dy, by);
            bz = fmaf(-hi, dz, bz);
        }
        if (k + 1 < k1) {                                          // take source (lane + k + 1)'s sum from the next lane
            const int from = (lane + 1) & 31;
            bx = __shfl_sync(0xffffffffu, bx, from);
            by = __shfl_sync(0xffffffffu, by, from);
            bz = __shfl_sync(0xffffffffu, bz, from);
        }
    }
    const int from = (lane - (k1 - 1)) & 31;                       // lane l now holds source (l + k1 - 1)'s sum
    bx = __shfl_sync(0xffffffffu, bx, from);
    by = __shfl_sync(0xffffffffu, by, from);
    bz = __shfl_sync(0xffffffffu, bz, from);
    if (lane < m) {
        atomicAdd(q.acc + src0 + lane, bx);
        atomicAdd(q.acc + q.n + src0 + lane, by);
        atomicAdd(q.acc + 2 * q.n + src0 + lane, bz);
    }
}

__global__ void __launch_bounds__(PP_WARPS * 32) k_pp_pairs(const PPArgs q) {
    __shared__ float4 sh[PP_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int M = q.M;
    const unsigned total = *q.n_items;
    float4* stage = sh[w];
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
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        // the item's own particles with each other (steps 1 .. 16)
        __syncwarp();
        stage[lane] = make_float4(tx, ty, tz, tm);
        __syncwarp();
        pp_chunk(stage, lane, 1, 17, true, tx, ty, tz, tm, q, ax, ay, az, t0, min(32, cl - t0));
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
                pp_chunk(stage, lane, 0, 32, false, tx, ty, tz, tm, q, ax, ay, az, j0, min(32, s1 - j0));
            }
        }
        if (act) {
            atomicAdd(q.acc + t, ax);
            atomicAdd(q.acc + q.n + t, ay);
            atomicAdd(q.acc + 2 * q.n + t, az);
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
    SSS_CUDA_TRY(ctx, sss_dev::radix_sort(k0, v0, k1, v1, n, (long long*)(B + o_rs), st, bits));
    k_pp_gather<<<blocks_for(n, 256), 256, 0, st>>>(parts, v0, src);
    SSS_LAUNCH_CHECK(ctx, "k_pp_gather");
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(first, 0, 4 * (size_t)cells, st));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(last, 0, 4 * (size_t)cells, st));
    k_pp_bounds<<<blocks_for(n, 256), 256, 0, st>>>(k0, n, first, last);
    SSS_LAUNCH_CHECK(ctx, "k_pp_bounds");
    k_pp_groups<<<blocks_for(cells, 256), 256, 0, st>>>(first, last, cells, groups);
    SSS_LAUNCH_CHECK(ctx, "k_pp_groups");
    SSS_CUDA_TRY(ctx, sss_dev::exclusive_scan(groups, offs, cells, (long long*)(B + o_rs), st));
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
