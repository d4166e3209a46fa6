// pm_sort.cu -- device-wide exclusive scan and stable LSD radix sort of
// (uint64 key, uint32 value) pairs.  They replace the CUDPP scan / compact /
// radix sort the reference builds its tree with (MNCudaPrimitives.cpp:160-227).
//
// Radix sort: 8-bit digits, reduce-then-scan per pass (no inter-block waits).
//   1. k_digit_hist: every tile counts its digits (one histogram per warp), in
//      the digit-major layout hist[d * tiles + t];
//   2. k_digit_rowscan: block d scans row d in place (the tile's offset among
//      the keys of digit d) and writes the row total (above 4M keys: one
//      exclusive scan of the whole array, which yields global offsets);
//   3. k_digit_scatter: every tile adds the exclusive scan of the 256 row
//      totals (the digit's start), ranks its keys stably, orders them by
//      digit in shared memory and writes each digit's run contiguously.
// Stability across passes makes the result sorted by the full key, with the
// input order breaking ties.
#include "pm_internal.h"

namespace pm {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;      // elements per thread per scan tile
constexpr int kScanTile = kScanThreads * kScanItems;

// ------------------------------------------------------------------ scan --

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
//
// One pass = k_digit_hist (per tile digit counts, digit-major so that one
// exclusive scan gives every tile its global offset per digit), the scan,
// and k_digit_scatter.  A tile is kSortTile keys; warp w of its block owns
// keys [w * 256, (w + 1) * 256) of the tile, taken in rounds of 32, so the
// order (warp, round, lane) is the input order.  The scatter ranks each key
// among the tile's keys of its digit (the lanes sharing its digit from eight
// ballots, plus per-warp digit counters), places the tile's keys sorted by digit in shared memory, and
// writes every digit's run out contiguously.

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 8;                                 // rounds of 32 keys per warp
constexpr int kSortTile = kSortThreads * kSortRounds;          // 2048 keys per tile

template <class Key>
__global__ void __launch_bounds__(kSortThreads) k_digit_hist(const Key* __restrict__ keys, uint32_t n,
                                                               int shift, uint32_t ntiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_hist[kSortWarps][256];   // one histogram per warp: contention only within a warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s_hist[w][threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile + (uint64_t)warp * (32 * kSortRounds);
    Key kk[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t g = base + (uint64_t)r * 32 + lane;
        kk[r] = g < n ? keys[g] : Key(0);
    }
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t g = base + (uint64_t)r * 32 + lane;
        if (g < n) atomicAdd(&s_hist[warp][(uint32_t)(kk[r] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) c += s_hist[w][threadIdx.x];
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = c;
}

// Block d: exclusive scan of hist[d * ntiles, (d + 1) * ntiles) in place,
// the row total to digit_total[d].
__global__ void __launch_bounds__(kScanThreads) k_digit_rowscan(uint32_t* __restrict__ hist, uint32_t ntiles,
                                                                 uint32_t* __restrict__ digit_total) {
    __shared__ uint32_t s_warp[32];
    uint32_t* row = hist + (size_t)blockIdx.x * ntiles;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < ntiles; base += kScanTile) {
        const uint32_t first = base + threadIdx.x * kScanItems;
        uint32_t v[kScanItems];
        uint32_t sum = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            v[i] = first + i < ntiles ? row[first + i] : 0u;
            sum += v[i];
        }
        uint32_t total;
        uint32_t run = carry + block_exclusive_scan(sum, s_warp, total);
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            if (first + i < ntiles) row[first + i] = run;
            run += v[i];
        }
        carry += total;
    }
    if (threadIdx.x == 0) digit_total[blockIdx.x] = carry;
}

// kGather (the build's last pass): instead of the values, the photons
// themselves go to their sorted positions (tree order), with the caller index
// in pos.w, the packed direction in pow.w, and the inverse permutation.
template <class Key, bool kGather>
__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const Key* __restrict__ keys_in,
                                                                  const uint32_t* __restrict__ vals_in, uint32_t n,
                                                                  int shift, uint32_t ntiles,
                                                                  const uint32_t* __restrict__ offsets,
                                                                  const uint32_t* __restrict__ digit_total,
                                                                  Key* __restrict__ keys_out,
                                                                  uint32_t* __restrict__ vals_out, SortGather gather) {
    __shared__ uint32_t s_cnt[kSortWarps][256];   // per-warp digit counts, then per-warp starts within the digit
    __shared__ uint32_t s_start[256];             // tile-local start of each digit
    __shared__ uint32_t s_global[256];            // global position of the tile's first key of each digit
    __shared__ uint32_t s_warpsum[32];
    __shared__ uint32_t s_warptot[32];
    __shared__ Key s_key[kSortTile];
    __shared__ uint32_t s_val[kSortTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s_cnt[w][threadIdx.x] = 0;
    // thread d: this tile's offset among the keys of digit d, and digit d's
    // row total (null: offsets are already global); used after the ranking
    const uint32_t toff = offsets[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    const uint32_t tot = digit_total ? digit_total[threadIdx.x] : 0u;
    __syncthreads();
    const uint64_t tile0 = (uint64_t)blockIdx.x * kSortTile;
    const uint64_t base = tile0 + (uint64_t)warp * (32 * kSortRounds);
    Key key[kSortRounds];
    uint32_t val[kSortRounds], rank[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t g = base + (uint64_t)r * 32 + lane;
        const bool valid = g < n;
        key[r] = valid ? keys_in[g] : Key(0);
        val[r] = valid ? vals_in[g] : 0u;
        const uint32_t digit = valid ? ((uint32_t)(key[r] >> shift) & 0xffu) : 256u;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);   // lanes with the same digit: 8 ballots
        if (!valid) peers = ~peers;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t ones = __ballot_sync(0xffffffffu, (digit >> b) & 1u);
            peers &= ((digit >> b) & 1u) ? ones : ~ones;
        }
        rank[r] = valid ? s_cnt[warp][digit] + __popc(peers & lt) : 0u;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) s_cnt[warp][digit] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {   // thread d: per-warp starts within digit d, then the tile-local digit starts
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = s_cnt[w][threadIdx.x];
            s_cnt[w][threadIdx.x] = run;
            run += c;
        }
        uint32_t x = run, y = tot;   // block exclusive scans: the tile's digit counts, the row totals
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t xo = __shfl_up_sync(0xffffffffu, x, o), yo = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) { x += xo; y += yo; }
        }
        if (lane == 31) { s_warpsum[warp] = x; s_warptot[warp] = y; }
        __syncthreads();
        uint32_t wp = 0, wt = 0;
        for (int w = 0; w < warp; ++w) { wp += s_warpsum[w]; wt += s_warptot[w]; }
        s_start[threadIdx.x] = wp + x - run;
        s_global[threadIdx.x] = wt + y - tot + toff;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t g = base + (uint64_t)r * 32 + lane;
        if (g < n) {
            const uint32_t digit = (uint32_t)(key[r] >> shift) & 0xffu;
            const uint32_t local = s_start[digit] + s_cnt[warp][digit] + rank[r];
            s_key[local] = key[r];
            s_val[local] = val[r];
        }
    }
    __syncthreads();
    const uint32_t tile_n = (uint32_t)min((uint64_t)kSortTile, (uint64_t)n - tile0);
    for (uint32_t i = threadIdx.x; i < tile_n; i += kSortThreads) {
        const Key kk = s_key[i];
        const uint32_t digit = (uint32_t)(kk >> shift) & 0xffu;
        const uint32_t dst = s_global[digit] + (i - s_start[digit]);
        keys_out[dst] = kk;
        if (kGather) {
            const uint32_t src = s_val[i];
            const float4 p = gather.in_pos[src];
            const float4 w = gather.in_pow[src];
            const uint32_t dir = (gather.format == 0) ? spherical_to_oct(p.w, w.w) : __float_as_uint(w.w);
            gather.out_pos[dst] = make_float4(p.x, p.y, p.z, __uint_as_float(src));
            gather.out_pow[dst] = make_float4(w.x, w.y, w.z, __uint_as_float(dir));
            gather.inv[src] = dst;
        } else {
            vals_out[dst] = s_val[i];
        }
    }
}

// Up to this many tiles (4M keys) a pass scans the digit rows with one
// launch of 256 blocks; above it a block walks its long row serially (a
// 3-pass sort of 67M pairs measured 0.27 ms slower with row scans), and the
// generic scan of the whole digit-major array (three launches, every SM
// busy) takes over.
constexpr uint32_t kRowScanMaxTiles = 2048;

size_t sort_scratch_words(uint32_t n) {
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    const size_t hist = (size_t)tiles * 256;   // per-tile digit counts
    return hist + (tiles <= kRowScanMaxTiles ? 256 : scan_scratch_words((uint32_t)hist) + 1);
}

// Sorts by bits [0, key_bits) of the keys.  Returns which buffer holds the
// result (0: keys[0]/vals[0], 1: keys[1]/vals[1]).  Buffers of the other
// index are clobbered.
template <class Key>
static int radix_sort_impl(Key* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                           cudaStream_t st, int* launches, const SortGather* gather) {
    if (n <= 1) return 0;
    int nl = 0;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* hist = scratch;
    uint32_t* tail = scratch + (size_t)tiles * 256;   // row totals, or the whole-array scan's scratch
    const bool rows = tiles <= kRowScanMaxTiles;
    int cur = 0;
    for (int shift = 0; shift < key_bits; shift += 8) {
        k_digit_hist<Key><<<tiles, kSortThreads, 0, st>>>(keys[cur], n, shift, tiles, hist);
        if (rows) {
            k_digit_rowscan<<<256, kScanThreads, 0, st>>>(hist, tiles, tail);
            nl += 3;
        } else {
            nl += 2 + exclusive_scan(hist, hist, tiles * 256u, tail, nullptr, st);
        }
        const uint32_t* dtot = rows ? tail : nullptr;
        if (gather && shift + 8 >= key_bits)
            k_digit_scatter<Key, true><<<tiles, kSortThreads, 0, st>>>(keys[cur], vals[cur], n, shift, tiles, hist,
                                                                       dtot, keys[cur ^ 1], vals[cur ^ 1], *gather);
        else
            k_digit_scatter<Key, false><<<tiles, kSortThreads, 0, st>>>(keys[cur], vals[cur], n, shift, tiles, hist,
                                                                        dtot, keys[cur ^ 1], vals[cur ^ 1], SortGather{});
        cur ^= 1;
    }
    if (launches) *launches += nl;
    return cur;
}

int radix_sort_pairs(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                     cudaStream_t st, int* launches, const SortGather* gather) {
    return radix_sort_impl<uint64_t>(keys, vals, n, key_bits, scratch, st, launches, gather);
}

int radix_sort_pairs32(uint32_t* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                       cudaStream_t st, int* launches) {
    return radix_sort_impl<uint32_t>(keys, vals, n, key_bits > 32 ? 32 : key_bits, scratch, st, launches, nullptr);
}

}  // namespace pm
