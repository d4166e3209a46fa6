// pm_sort.cu -- device-wide exclusive scan and stable LSD radix sort of
// (uint64 key, uint32 value) pairs.  They replace the CUDPP scan / compact /
// radix sort the reference builds its tree with (MNCudaPrimitives.cpp:160-227).
//
// Radix sort: 8-bit digits, reduce-then-scan per pass.
//   1. k_digit_hist: every tile of kTile keys counts its digits
//      (digit-major layout hist[d * tiles + t], so one exclusive scan over
//      the whole array yields every tile's global offset per digit);
//   2. exclusive scan of hist;
//   3. k_digit_scatter: every tile ranks its keys stably (warp match_any +
//      per-warp digit counts) and scatters them to offset + rank.
// Stability across passes makes the result sorted by the full key, with the
// input order breaking ties.
#include "pm_internal.h"

namespace pm {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;      // elements per thread per scan tile
constexpr int kScanTile = kScanThreads * kScanItems;

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;   // 4096 keys per tile
constexpr int kSortWarps = kSortThreads / 32;

// ------------------------------------------------------------------ scan --

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < nwarps) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nwarps) s_warp[lane] = w;
    }
    __syncthreads();
    total = s_warp[nwarps - 1];
    const uint32_t warp_prefix = warp ? s_warp[warp - 1] : 0u;
    __syncthreads();
    return warp_prefix + x - v;
}

// Per-tile sums of in[0, n).
__global__ void k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t s_warp[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    uint32_t v = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint64_t g = base + (uint64_t)i * kScanThreads + threadIdx.x;
        if (g < n) v += in[g];
    }
    uint32_t total;
    block_exclusive_scan(v, s_warp, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Exclusive scan of tile_sums in place by one block (sequential over chunks);
// writes the grand total to *total_out when non-null.
__global__ void k_scan_tiles(uint32_t* __restrict__ tile_sums, uint32_t ntiles, uint32_t* __restrict__ total_out) {
    __shared__ uint32_t s_warp[32];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < ntiles; base += blockDim.x) {
        const uint32_t g = base + threadIdx.x;
        const uint32_t v = (g < ntiles) ? tile_sums[g] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(v, s_warp, total);
        if (g < ntiles) tile_sums[g] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

// out[i] = exclusive prefix of in (in and out may alias).
__global__ void k_scan_apply(const uint32_t* in, uint32_t n, const uint32_t* __restrict__ tile_offsets, uint32_t* out) {
    __shared__ uint32_t s_warp[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint64_t g = base + i;
        v[i] = (g < n) ? in[g] : 0u;
        sum += v[i];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, s_warp, total) + tile_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint64_t g = base + i;
        if (g < n) out[g] = run;
        run += v[i];
    }
}

size_t scan_scratch_words(uint32_t n) { return (size_t)(n + kScanTile - 1) / kScanTile + 1; }

int exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, uint32_t* total_out,
                   cudaStream_t st) {
    if (n == 0) {
        if (total_out) cudaMemsetAsync(total_out, 0, sizeof(uint32_t), st);
        return 0;
    }
    const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    k_scan_reduce<<<tiles, kScanThreads, 0, st>>>(in, n, scratch);
    k_scan_tiles<<<1, kScanThreads, 0, st>>>(scratch, tiles, total_out);
    k_scan_apply<<<tiles, kScanThreads, 0, st>>>(in, n, scratch, out);
    return 3;
}

// ------------------------------------------------------------ radix sort --

template <class Key>
__global__ void __launch_bounds__(kSortThreads) k_digit_hist(const Key* __restrict__ keys, uint32_t n,
                                                               int shift, uint32_t ntiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_hist[256];
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int i = 0; i < kSortItems; ++i) {
        const uint64_t g = base + (uint64_t)i * kSortThreads + threadIdx.x;
        if (g < n) atomicAdd(&s_hist[(uint32_t)(keys[g] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = s_hist[threadIdx.x];
}

template <class Key>
__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const Key* __restrict__ keys_in,
                                                                  const uint32_t* __restrict__ vals_in, uint32_t n,
                                                                  int shift, uint32_t ntiles,
                                                                  const uint32_t* __restrict__ offsets,
                                                                  Key* __restrict__ keys_out,
                                                                  uint32_t* __restrict__ vals_out) {
    __shared__ uint32_t s_base[256];              // global offset + keys of this digit seen so far
    __shared__ uint32_t s_warp[kSortWarps][256];  // per-warp count, then per-warp start
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_base[threadIdx.x] = offsets[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int i = 0; i < kSortItems; ++i) {
        const uint64_t g = base + (uint64_t)i * kSortThreads + threadIdx.x;
        const bool valid = g < n;
        Key key = valid ? keys_in[g] : Key(0);
        uint32_t val = valid ? vals_in[g] : 0u;
        const uint32_t digit = valid ? ((uint32_t)(key >> shift) & 0xffu) : 256u;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) s_warp[w][threadIdx.x] = 0;
        __syncthreads();
        const uint32_t peers = __match_any_sync(0xffffffffu, digit);
        const uint32_t rank_in_warp = __popc(peers & lt_mask);
        if (valid && rank_in_warp == 0) s_warp[warp][digit] = __popc(peers);
        __syncthreads();
        {   // thread d: turn per-warp counts for digit d into start offsets
            uint32_t run = s_base[threadIdx.x];
#pragma unroll
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t c = s_warp[w][threadIdx.x];
                s_warp[w][threadIdx.x] = run;
                run += c;
            }
            s_base[threadIdx.x] = run;
        }
        __syncthreads();
        if (valid) {
            const uint32_t dst = s_warp[warp][digit] + rank_in_warp;
            keys_out[dst] = key;
            vals_out[dst] = val;
        }
        __syncthreads();
    }
}

size_t sort_scratch_words(uint32_t n) {
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    const size_t hist = (size_t)tiles * 256;
    return hist + scan_scratch_words((uint32_t)hist) + 1;
}

// Sorts by bits [0, key_bits) of the keys.  Returns which buffer holds the
// result (0: keys[0]/vals[0], 1: keys[1]/vals[1]).  Buffers of the other
// index are clobbered.
template <class Key>
static int radix_sort_impl(Key* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                           cudaStream_t st, int* launches) {
    if (n <= 1) return 0;
    int nl = 0;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* hist = scratch;
    uint32_t* scan_tmp = scratch + (size_t)tiles * 256;
    int cur = 0;
    for (int shift = 0; shift < key_bits; shift += 8) {
        k_digit_hist<Key><<<tiles, kSortThreads, 0, st>>>(keys[cur], n, shift, tiles, hist);
        nl += 2 + exclusive_scan(hist, hist, tiles * 256u, scan_tmp, nullptr, st);
        k_digit_scatter<Key><<<tiles, kSortThreads, 0, st>>>(keys[cur], vals[cur], n, shift, tiles, hist,
                                                              keys[cur ^ 1], vals[cur ^ 1]);
        cur ^= 1;
    }
    if (launches) *launches += nl;
    return cur;
}

int radix_sort_pairs(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                     cudaStream_t st, int* launches) {
    return radix_sort_impl<uint64_t>(keys, vals, n, key_bits, scratch, st, launches);
}

int radix_sort_pairs32(uint32_t* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                       cudaStream_t st, int* launches) {
    return radix_sort_impl<uint32_t>(keys, vals, n, key_bits > 32 ? 32 : key_bits, scratch, st, launches);
}

}  // namespace pm
