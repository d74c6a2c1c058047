// Device-wide exclusive prefix sums (int64) and a stable LSD radix sort of
// 64-bit keys with 32-bit values, written for the broadphase. All launches go
// to one stream; temporary storage comes from the caller.
#pragma once

#include "sss_internal.cuh"

namespace sss_dev {
// internal linkage: every translation unit that includes this header gets its own copy of the kernels
namespace {

constexpr int SCAN_NT = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_NT * SCAN_ITEMS;   // 2048 elements per block

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* total) {
    __shared__ long long s_warp[SCAN_NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        long long w = (lane < SCAN_NT / 32) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_NT / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const long long before = (warp > 0 ? s_warp[warp - 1] : 0) + x - v;
    *total = s_warp[SCAN_NT / 32 - 1];
    __syncthreads();
    return before;
}

// per-block sums of int64 input
__global__ void __launch_bounds__(SCAN_NT) k_tile_sums(const long long* __restrict__ in, long long n,
                                                       long long* __restrict__ sums) {
    const long long base = (long long)blockIdx.x * SCAN_TILE;
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + (long long)k * SCAN_NT + threadIdx.x;
        if (i < n) s += in[i];
    }
    long long tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// exclusive scan of `n` sums in one block (any n), total into sums[n]
__global__ void __launch_bounds__(SCAN_NT) k_scan_sums(long long* __restrict__ sums, long long n) {
    long long carry = 0;
    for (long long b = 0; b < n; b += SCAN_NT) {
        const long long i = b + threadIdx.x;
        const long long v = i < n ? sums[i] : 0;
        long long tot;
        const long long ex = block_exclusive_scan(v, &tot);
        if (i < n) sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) sums[n] = carry;
}

// out[i] = exclusive prefix of in (in-place allowed); thread-ordered tiles
__global__ void __launch_bounds__(SCAN_NT) k_tile_scan(const long long* __restrict__ in, long long n,
                                                       const long long* __restrict__ offs, long long* out) {
    const long long base = (long long)blockIdx.x * SCAN_TILE;
    long long v[SCAN_ITEMS];
    long long s = 0;
    // each thread scans SCAN_ITEMS consecutive elements
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    long long tot;
    long long run = block_exclusive_scan(s, &tot) + offs[blockIdx.x];
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

// Scratch (long long elements) an exclusive scan of n elements needs.
inline size_t scan_scratch(long long n) { return (size_t)((n + SCAN_TILE - 1) / SCAN_TILE) + 1; }

// Exclusive scan of n int64 into out (may alias in); *total_dev receives the sum.
inline cudaError_t exclusive_scan(const long long* in, long long* out, long long n, long long* scratch,
                                  cudaStream_t s) {
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 0) {
        return cudaMemsetAsync(scratch, 0, sizeof(long long), s);
    }
    k_tile_sums<<<(unsigned)tiles, SCAN_NT, 0, s>>>(in, n, scratch);
    k_scan_sums<<<1, SCAN_NT, 0, s>>>(scratch, tiles);
    k_tile_scan<<<(unsigned)tiles, SCAN_NT, 0, s>>>(in, n, scratch, out);
    return cudaGetLastError();
}
// total of the last exclusive_scan: scratch[tiles]

// ----------------------------------------------------------- radix sort

constexpr int RS_NT = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_NT * RS_ITEMS;
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;

__device__ __forceinline__ unsigned digit_of(unsigned long long k, int shift) {
    return (unsigned)(k >> shift) & (RS_BINS - 1);
}

// hist[d * n_tiles + tile] = count of digit d in the tile
__global__ void __launch_bounds__(RS_NT) k_rs_hist(const unsigned long long* __restrict__ keys, long long n,
                                                   int shift, long long* __restrict__ hist, int n_tiles) {
    __shared__ unsigned cnt[RS_BINS];
    for (int d = threadIdx.x; d < RS_BINS; d += RS_NT) cnt[d] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; ++k) {
        const long long i = base + (long long)k * RS_NT + threadIdx.x;
        if (i < n) atomicAdd(&cnt[digit_of(keys[i], shift)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RS_BINS; d += RS_NT) hist[(long long)d * n_tiles + blockIdx.x] = cnt[d];
}

// Stable scatter: elements of a tile are ranked in their original order
// (rounds of RS_NT consecutive elements; warp match + per-warp digit counts).
__global__ void __launch_bounds__(RS_NT) k_rs_scatter(const unsigned long long* __restrict__ keys_in,
                                                      const unsigned* __restrict__ vals_in, long long n, int shift,
                                                      const long long* __restrict__ offs, int n_tiles,
                                                      unsigned long long* __restrict__ keys_out,
                                                      unsigned* __restrict__ vals_out) {
    constexpr int NW = RS_NT / 32;
    __shared__ unsigned s_wcnt[NW][RS_BINS];
    __shared__ long long s_base[RS_BINS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < RS_BINS; d += RS_NT) s_base[d] = offs[(long long)d * n_tiles + blockIdx.x];
    const unsigned lt = (1u << lane) - 1u;
    const long long base = (long long)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; ++k) {
        for (int t = threadIdx.x; t < NW * RS_BINS; t += RS_NT) (&s_wcnt[0][0])[t] = 0;
        __syncthreads();
        const long long i = base + (long long)k * RS_NT + threadIdx.x;
        const bool valid = i < n;
        unsigned long long key = 0;
        unsigned val = 0, d = RS_BINS;    // RS_BINS = no element
        if (valid) {
            key = keys_in[i];
            val = vals_in[i];
            d = digit_of(key, shift);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & lt);
        if (valid && rank == 0) s_wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            long long pos = s_base[d] + rank;
            for (int w = 0; w < warp; ++w) pos += s_wcnt[w][d];
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        for (int dd = threadIdx.x; dd < RS_BINS; dd += RS_NT) {
            unsigned add = 0;
            for (int w = 0; w < NW; ++w) add += s_wcnt[w][dd];
            s_base[dd] += add;
        }
        __syncthreads();
    }
}

// Scratch (long long elements) radix_sort needs for n elements.
inline size_t radix_scratch(long long n) {
    const long long tiles = (n + RS_TILE - 1) / RS_TILE;
    return (size_t)(tiles * RS_BINS) + scan_scratch(tiles * RS_BINS);
}

// Stable ascending sort of unsigned 64-bit keys with values, on the low
// `bits` bits of the keys (the higher bits must be zero; rounded up to an
// even number of 8-bit passes). keys/vals are sorted through the alternate
// buffers; the result ends in (k0, v0).
inline cudaError_t radix_sort(unsigned long long* k0, unsigned* v0, unsigned long long* k1, unsigned* v1,
                              long long n, long long* scratch, cudaStream_t s, int bits = 64) {
    if (n <= 1) return cudaSuccess;
    const int tiles = (int)((n + RS_TILE - 1) / RS_TILE);
    long long* hist = scratch;
    long long* scan_tmp = scratch + (size_t)tiles * RS_BINS;
    const int want = (bits + 2 * RS_BITS - 1) / (2 * RS_BITS) * 2;
    const int passes = want < 64 / RS_BITS ? want : 64 / RS_BITS;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = pass * RS_BITS;
        unsigned long long* kin = (pass & 1) ? k1 : k0;
        unsigned* vin = (pass & 1) ? v1 : v0;
        unsigned long long* kout = (pass & 1) ? k0 : k1;
        unsigned* vout = (pass & 1) ? v0 : v1;
        k_rs_hist<<<tiles, RS_NT, 0, s>>>(kin, n, shift, hist, tiles);
        cudaError_t e = exclusive_scan(hist, hist, (long long)tiles * RS_BINS, scan_tmp, s);
        if (e != cudaSuccess) return e;
        k_rs_scatter<<<tiles, RS_NT, 0, s>>>(kin, vin, n, shift, hist, tiles, kout, vout);
    }
    return cudaGetLastError();   // an even number of passes: the result is back in (k0, v0)
}

}  // namespace
}  // namespace sss_dev
