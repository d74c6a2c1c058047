// Device-wide exclusive prefix sums (int64) and a stable LSD radix sort of
// 64-bit keys with 32-bit values, both single-pass with decoupled look-back.
// All launches go to one stream; temporary storage comes from the caller.
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

// Bounded spin on a word another block publishes: true once *p satisfies
// ready(*p); false (and SSS_ERR_TIMEOUT in *err) after SSS_WAIT_LIMIT_NS. The
// blocks waited on took their tile numbers earlier (an atomic ticket), so they
// are running or done and the wait ends.
template <typename T, typename F>
__device__ __forceinline__ bool spin_until(const volatile T* p, T& v, F ready, int* err) {
    v = *p;
    if (ready(v)) return true;
    const uint64_t t0 = sss_globaltimer();
    for (;;) {
        v = *p;
        if (ready(v)) return true;
        if (sss_globaltimer() - t0 > SSS_WAIT_LIMIT_NS) {
            if (err) atomicExch(err, SSS_ERR_TIMEOUT);
            return false;
        }
    }
}

// Single-pass exclusive scan (decoupled look-back, Merrill & Garland 2016):
// a block takes the next tile by ticket, scans it (each thread SCAN_ITEMS
// consecutive elements), publishes the tile's sum, finds the sum of all
// tiles before it by walking back over the published sums (a tile's
// inclusive prefix ends the walk), publishes its own inclusive prefix and
// writes its outputs. Scratch (long long): total at [tiles], then the
// ticket, then per tile the sum, the inclusive prefix and a flag word.
struct ScanState {
    long long* total;
    unsigned* ticket;
    long long* agg;
    long long* inc;
    int* flag;            // 0 none, 1 sum published, 2 inclusive prefix published
};

__global__ void __launch_bounds__(SCAN_NT) k_scan_1pass(const long long* in, long long n, long long* out,
                                                         ScanState st, long long tiles, int* err) {
    __shared__ unsigned s_tile;
    __shared__ long long s_excl;
    if (threadIdx.x == 0) s_tile = atomicAdd(st.ticket, 1u);
    __syncthreads();
    const long long tile = s_tile;
    const long long base = tile * SCAN_TILE;
    long long v[SCAN_ITEMS];
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    long long tot;
    long long run = block_exclusive_scan(s, &tot);
    if (threadIdx.x < 32) {
        // warp 0 walks back 32 tiles at a time: lane l reads tile pos - l; the
        // nearest tile with its inclusive prefix published ends the walk
        const int lane = threadIdx.x;
        long long excl = 0;
        if (tile > 0) {
            if (lane == 0) {
                st.agg[tile] = tot;
                __threadfence();
                atomicExch(&st.flag[tile], 1);
            }
            for (long long pos = tile - 1;; pos -= 32) {
                const long long idx = pos - lane;
                int f = 2;                      // before tile 0: an inclusive prefix of 0
                long long val = 0;
                if (idx >= 0) {
                    if (spin_until<int>(st.flag + idx, f, [](int q) { return q != 0; }, err)) {
                        __threadfence();
                        val = (f == 2) ? *(volatile long long*)(st.inc + idx) : *(volatile long long*)(st.agg + idx);
                    } else {
                        f = 2;                  // timed out (status set): stop here
                    }
                }
                const unsigned incm = __ballot_sync(0xffffffffu, f == 2);
                const int first = incm ? __ffs(incm) - 1 : 32;
                if (lane > first) val = 0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
                excl += val;
                if (incm) break;
            }
        }
        if (lane == 0) {
            st.inc[tile] = excl + tot;
            __threadfence();
            atomicExch(&st.flag[tile], 2);
            if (tile == tiles - 1) *st.total = excl + tot;
            s_excl = excl;
        }
    }
    __syncthreads();
    run += s_excl;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

// Scratch (long long elements) an exclusive scan of n elements needs.
inline size_t scan_scratch(long long n) {
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    return (size_t)(tiles + 1) + 1 + 2 * (size_t)tiles + (size_t)(tiles + 1) / 2;
}

// Exclusive scan of n int64 into out (may alias in); the total goes to
// scratch[tiles] (tiles = ceil(n / SCAN_TILE)). Two stream operations: a
// clear of the ticket and flags, the scan kernel.
inline cudaError_t exclusive_scan(const long long* in, long long* out, long long n, long long* scratch,
                                  cudaStream_t s, int* err) {
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 0) {
        return cudaMemsetAsync(scratch, 0, sizeof(long long), s);
    }
    ScanState st;
    st.total = scratch + tiles;
    st.ticket = reinterpret_cast<unsigned*>(scratch + tiles + 1);
    st.agg = scratch + tiles + 2;
    st.inc = st.agg + tiles;
    st.flag = reinterpret_cast<int*>(st.inc + tiles);
    cudaError_t e = cudaMemsetAsync(st.ticket, 0, sizeof(long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(st.flag, 0, (size_t)tiles * sizeof(int), s);
    if (e != cudaSuccess) return e;
    k_scan_1pass<<<(unsigned)tiles, SCAN_NT, 0, s>>>(in, n, out, st, tiles, err);
    return cudaGetLastError();
}

// ----------------------------------------------------------- radix sort
//
// Stable LSD radix sort of 64-bit keys with 32-bit values, 8-bit digits,
// one kernel per digit pass (Adinets & Merrill, "Onesweep", 2022): one
// launch counts the digits of every pass over all keys; each pass kernel
// takes a tile by ticket, ranks its keys stably, publishes its digit counts,
// looks back over the tiles before it for each digit's exclusive prefix (as
// the scan above, one digit per thread) and scatters. A pass whose digit is
// the same for every key is a copy.

constexpr int RS_NT = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_NT * RS_ITEMS;
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;
constexpr int RS_MAX_PASSES = 64 / RS_BITS;
static_assert(RS_BINS == RS_NT, "one digit per thread in the look-back");

constexpr unsigned long long RS_FLAG_AGG = 1ull << 62, RS_FLAG_INC = 2ull << 62, RS_VAL = (1ull << 62) - 1;

__device__ __forceinline__ unsigned digit_of(unsigned long long k, int shift) {
    return (unsigned)(k >> shift) & (RS_BINS - 1);
}

// hist[p][d] += count of digit d of pass p over all keys
__global__ void __launch_bounds__(RS_NT) k_rs_hist_all(const unsigned long long* __restrict__ keys, long long n,
                                                      int passes, unsigned long long* __restrict__ hist) {
    __shared__ unsigned cnt[RS_MAX_PASSES][RS_BINS];
    for (int i = threadIdx.x; i < RS_MAX_PASSES * RS_BINS; i += RS_NT) (&cnt[0][0])[i] = 0;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * RS_NT + threadIdx.x; i < n; i += (long long)gridDim.x * RS_NT) {
        const unsigned long long k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&cnt[p][digit_of(k, p * RS_BITS)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RS_BINS; i += RS_NT) {
        const unsigned c = (&cnt[0][0])[i];
        if (c) atomicAdd(&hist[i], (unsigned long long)c);
    }
}

__global__ void __launch_bounds__(RS_NT) k_rs_pass(const unsigned long long* __restrict__ keys_in,
                                                  const unsigned* __restrict__ vals_in, long long n, int shift,
                                                  const unsigned long long* __restrict__ hist, unsigned* ticket,
                                                  unsigned long long* status,
                                                  unsigned long long* __restrict__ keys_out,
                                                  unsigned* __restrict__ vals_out, int* err) {
    constexpr int NW = RS_NT / 32;
    __shared__ unsigned s_wcnt[NW][RS_BINS];
    __shared__ long long s_base[RS_BINS];
    __shared__ unsigned s_cnt[RS_BINS];
    __shared__ unsigned s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(ticket, 1u);
    s_cnt[tid] = 0;
    __syncthreads();
    const long long tile = s_tile;
    const long long base = tile * RS_TILE;
    const unsigned long long hc = hist[tid];
    long long tot;
    const long long goff = block_exclusive_scan((long long)hc, &tot);   // digit tid's first output position
    const bool trivial = __syncthreads_or(hc == (unsigned long long)n);
    unsigned long long key[RS_ITEMS];
    unsigned val[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const long long i = base + (long long)k * RS_NT + tid;
        key[k] = i < n ? keys_in[i] : 0ull;
        val[k] = i < n ? vals_in[i] : 0u;
    }
    if (trivial) {   // every key has the same digit: the pass keeps the order
#pragma unroll
        for (int k = 0; k < RS_ITEMS; ++k) {
            const long long i = base + (long long)k * RS_NT + tid;
            if (i < n) {
                keys_out[i] = key[k];
                vals_out[i] = val[k];
            }
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k)
        if (base + (long long)k * RS_NT + tid < n) atomicAdd(&s_cnt[digit_of(key[k], shift)], 1u);
    __syncthreads();
    // digit tid: publish this tile's count, look back for the count before it
    const unsigned long long c = s_cnt[tid];
    unsigned long long excl = 0;
    volatile unsigned long long* mine = status + tile * RS_BINS + tid;
    if (tile > 0) {
        *mine = c | RS_FLAG_AGG;
        for (long long t = tile - 1; t >= 0; --t) {
            unsigned long long w;
            if (!spin_until<unsigned long long>(status + t * RS_BINS + tid, w,
                                                [](unsigned long long q) { return (q >> 62) != 0; }, err))
                break;
            excl += w & RS_VAL;
            if ((w >> 62) == 2) break;
        }
    }
    *mine = (excl + c) | RS_FLAG_INC;
    s_base[tid] = goff + (long long)excl;
    const unsigned lt = (1u << lane) - 1u;
    for (int k = 0; k < RS_ITEMS; ++k) {
        for (int t = tid; t < NW * RS_BINS; t += RS_NT) (&s_wcnt[0][0])[t] = 0;
        __syncthreads();
        const long long i = base + (long long)k * RS_NT + tid;
        const bool valid = i < n;
        const unsigned d = valid ? digit_of(key[k], shift) : RS_BINS;   // RS_BINS = no element
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & lt);
        if (valid && rank == 0) s_wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            long long pos = s_base[d] + rank;
            for (int w = 0; w < warp; ++w) pos += s_wcnt[w][d];
            keys_out[pos] = key[k];
            vals_out[pos] = val[k];
        }
        __syncthreads();
        {
            unsigned add = 0;
            for (int w = 0; w < NW; ++w) add += s_wcnt[w][tid];
            s_base[tid] += add;
        }
    }
}

// Scratch (long long elements) radix_sort needs for n elements.
inline size_t radix_scratch(long long n) {
    const long long tiles = (n + RS_TILE - 1) / RS_TILE;
    return (size_t)RS_MAX_PASSES * RS_BINS + 8 + (size_t)RS_MAX_PASSES * (size_t)tiles * RS_BINS;
}

// Stable ascending sort of unsigned 64-bit keys with values, on the low
// `bits` bits of the keys (the higher bits must be zero; rounded up to an
// even number of 8-bit passes). keys/vals are sorted through the alternate
// buffers; the result ends in (k0, v0). A timed-out look-back sets
// SSS_ERR_TIMEOUT in *err.
inline cudaError_t radix_sort(unsigned long long* k0, unsigned* v0, unsigned long long* k1, unsigned* v1,
                              long long n, long long* scratch, cudaStream_t s, int* err, int bits = 64) {
    if (n <= 1) return cudaSuccess;
    const long long tiles = (n + RS_TILE - 1) / RS_TILE;
    const int want = (bits + 2 * RS_BITS - 1) / (2 * RS_BITS) * 2;
    const int passes = want < RS_MAX_PASSES ? want : RS_MAX_PASSES;
    unsigned long long* hist = reinterpret_cast<unsigned long long*>(scratch);
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + RS_MAX_PASSES * RS_BINS);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(scratch + RS_MAX_PASSES * RS_BINS + 8);
    cudaError_t e = cudaMemsetAsync(scratch, 0,
                                    ((size_t)RS_MAX_PASSES * RS_BINS + 8 + (size_t)passes * tiles * RS_BINS) *
                                        sizeof(long long), s);
    if (e != cudaSuccess) return e;
    const long long hb = tiles < 1024 ? tiles : 1024;
    k_rs_hist_all<<<(unsigned)hb, RS_NT, 0, s>>>(k0, n, passes, hist);
    for (int pass = 0; pass < passes; ++pass) {
        unsigned long long* kin = (pass & 1) ? k1 : k0;
        unsigned* vin = (pass & 1) ? v1 : v0;
        unsigned long long* kout = (pass & 1) ? k0 : k1;
        unsigned* vout = (pass & 1) ? v0 : v1;
        k_rs_pass<<<(unsigned)tiles, RS_NT, 0, s>>>(kin, vin, n, pass * RS_BITS, hist + pass * RS_BINS,
                                                    ticket + pass, status + (size_t)pass * tiles * RS_BINS, kout,
                                                    vout, err);
    }
    return cudaGetLastError();   // an even number of passes: the result is back in (k0, v0)
}

}  // namespace
}  // namespace sss_dev
