// pm_internal.h -- declarations shared by the engine's translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "pm_common.cuh"

namespace pm {

// ------------------------------------------------ device-side helpers --

// Exclusive scan of one value per thread over the block (blockDim.x a
// multiple of 32, at most 1024); total = the block's sum.  s_warp: 32 words
// of shared memory.
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

// Relaxed 64-bit loads and stores of the look-back words (status and value
// in one word, so no other data is ordered by them).
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Polls of one look-back word before a wait gives up (sets kErrWait).
constexpr uint32_t kLookbackWaitLimit = 1u << 22;

// Decoupled look-back over one value per tile (D. Merrill and M. Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016), called
// by all 32 lanes of one warp of the block that holds tile `tile`.  The tile
// publishes its aggregate; lane l then reads the word of tile base - l, 32
// earlier tiles per step, waits until all 32 have published, and adds their
// values up to the nearest one holding an inclusive prefix (or all 32
// aggregates, then the next 32).  The tile publishes its own inclusive
// prefix; every lane returns the exclusive prefix.  words: one uint64 per
// tile, cleared before the launch; status in bits 62-63 (1 aggregate, 2
// inclusive prefix).  Tiles must be taken in the order blocks start (an
// atomic ticket), so that a tile only waits for tiles whose blocks are
// running and publish their aggregates before they wait themselves.
__device__ __forceinline__ uint64_t warp_lookback_exclusive(uint64_t* words, uint32_t tile, uint64_t agg,
                                                            uint32_t* err) {
    constexpr uint64_t kAgg = 1ull << 62, kPrefix = 2ull << 62, kValue = (1ull << 62) - 1ull;
    const uint32_t lane = threadIdx.x & 31u;
    if (tile == 0) {
        if (lane == 0) st_relaxed_u64(words, kPrefix | agg);
        return 0;
    }
    if (lane == 0) st_relaxed_u64(words + tile, kAgg | agg);
    uint64_t before = 0;
    int64_t base = (int64_t)tile - 1;
    uint32_t polls = 0;
    for (;;) {
        const int64_t t = base - (int64_t)lane;
        uint64_t w = t >= 0 ? ld_relaxed_u64(words + t) : kPrefix;   // before tile 0: a zero prefix
        bool gave_up = false;
        while (__any_sync(0xffffffffu, (w >> 62) == 0)) {
            if (++polls > kLookbackWaitLimit) { gave_up = true; break; }   // never expected
            if (polls > 32) __nanosleep(64);
            if ((w >> 62) == 0) w = ld_relaxed_u64(words + t);
        }
        if (gave_up) {
            if (lane == 0 && err) atomicOr(err, kErrWait);
            break;
        }
        const uint32_t pm = __ballot_sync(0xffffffffu, (w >> 62) == 2);
        uint64_t v = w & kValue;
        if (pm && lane > (uint32_t)(__ffs(pm) - 1)) v = 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        before += v;
        if (pm) break;
        base -= 32;
    }
    if (lane == 0) st_relaxed_u64(words + tile, kPrefix | (before + agg));
    return before;
}

// pm_sort.cu
size_t scan_scratch_words(uint32_t n);
int exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, uint32_t* total_out,
                   cudaStream_t st);
size_t sort_scratch_words(uint32_t n);
struct SortGather {   // the last pass moves the photons, not the values (n >= 2 only)
    const float4* in_pos;
    const float4* in_pow;
    int format;           // PM_PHOTONS_*: 0 = reference angles, converted to the packed direction
    float4* out_pos;      // tree order: xyz, w = caller index bits
    float4* out_pow;      // tree order: rgb, w = packed direction
    uint32_t* inv;        // caller index -> tree position
};
int radix_sort_pairs(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                     cudaStream_t st, int* launches = nullptr, const SortGather* gather = nullptr);
int radix_sort_pairs32(uint32_t* keys[2], uint32_t* vals[2], uint32_t n, int key_bits, uint32_t* scratch,
                       cudaStream_t st, int* launches = nullptr);

// One photon map of a batch: geometry written by the batch build, query
// parameters uploaded by the host.
struct __align__(16) BatchGeom {
    ChildSlot root;        // slot of the map's subtree (empty slot for an empty map)
    ChildSlot wroot;       // the same subtree in the 32-wide tree
    float lo[3];           // photon bounds, lower corner
    float mscale;          // Morton scale of the map's cubic cell
    float fix_scale;       // fix_scale_of(largest flux channel)
    float max_power;
    uint32_t pad[2];
};
struct __align__(16) BatchQuery {
    uint32_t q_off, q_n;   // queries [q_off, q_off + q_n) of the batch
    uint32_t ph_off, ph_n; // photons [ph_off, ph_off + ph_n) of the batch
    uint64_t nbr_off;      // first neighbour slot of the map's rows (rows hold k entries)
    uint32_t k, min_found;
    float r2max, rmax, cone_k;
    int filter;
    double norm_c;         // filter normalisation constant (the estimate's factor is norm_c / r^2)
};

// Device buffers describing one built map (the build writes them, the
// query reads them).  Pointers are device addresses.
struct MapView {
    const float4* pos;      // tree order: xyz, w = caller index bits
    const float4* pow;      // tree order: rgb, w = octahedral direction bits
    const uint32_t* inv;    // caller index -> tree position
    const Node* nodes;      // [0] = super-root, internal nodes from 1
    const ChildSlot* wchild;   // 32-wide tree: child slots
    const ChildSlot* wroot;    // 32-wide tree: start slot
    MapHeader* hdr;
    uint32_t n;             // photon count (host copy)
};

struct BuildBuffers {
    uint64_t* keys[2];
    uint32_t* vals[2];
    uint32_t* scratch;      // sort / scan scratch
    uint32_t* kfirst;       // Karras internal nodes: first, last, split
    uint32_t* klast;
    uint32_t* ksplit;
    uint32_t* kkeep;        // keep flag (node holds more than leaf_size photons)
    uint32_t* krank;        // exclusive scan of kkeep = compacted index - 1
    uint32_t* parent;       // compacted node -> parent (node << 1 | side)
    uint32_t* arrive;       // refit arrival counters per compacted node
    uint32_t* nleaf;        // leaf children per compacted node
    uint32_t* partials;     // bounds reduction partials (block count * 8 floats) + counter
    uint32_t num_partials;
};

struct WideBuffers {
    uint32_t* wflag;       // per compacted node: is a wide node
    uint32_t* wcnt;        // per wide node: child count
    uint32_t* wfirst;      // scan of wcnt: first child slot
    ChildSlot* wchild;     // child slots of all wide nodes
    ChildSlot* wroot;      // start slot of the wide traversal
    uint32_t* scratch;     // child-count scan: ticket, total, look-back words (wide_scan_words)
};

// pm_build.cu
size_t build_bytes_needed(uint32_t n);
size_t wide_scan_words(uint32_t n);   // WideBuffers::scratch
// Returns the number of kernels launched; sort_done (if set) is recorded on
// the stream right after the radix sort.
// The whole single-map build, binary and 32-wide tree.
int build_map(const float4* in_pos, const float4* in_pow, uint32_t n, int format, uint32_t leaf_size,
              float4* out_pos, float4* out_pow, uint32_t* inv, Node* nodes, MapHeader* hdr, const BuildBuffers& bb,
              const WideBuffers& wide, cudaStream_t st, cudaEvent_t sort_done = nullptr);
void scale_flux(float4* pow, uint32_t n, float scale, MapHeader* hdr, cudaStream_t st);
int build_wide(uint32_t n, const Node* nodes, const uint32_t* parent, const uint32_t* rootmark, MapHeader* hdr,
               const WideBuffers& wb, cudaStream_t st);
int build_from_sorted(const float4* in_pos, const float4* in_pow, uint32_t n, int format, uint32_t leaf_size,
                      const uint64_t* keys, const uint32_t* vals, float4* out_pos, float4* out_pow, uint32_t* inv,
                      Node* nodes, MapHeader* hdr, const BuildBuffers& bb, cudaStream_t st, bool gathered = false,
                      const WideBuffers* wide = nullptr);   // wide: also the 32-wide tree (single map, n >= 2)

// pm_query.cu
struct QueryParams {
    uint32_t k;
    float r;             // R
    float r2;            // R^2 rounded in FP32
    int filter;
    float cone_k;
    uint32_t min_found;
};

struct QueryOutputs {
    float4* rad;         // required
    uint32_t* nbr;       // optional
    float* r2;           // optional
    uint32_t* count;     // optional
};

int query_order_keys(const float4* qpos, uint32_t nq, const MapHeader* hdr, uint32_t* keys, uint32_t* vals,
                       cudaStream_t st, bool hilbert = true);
constexpr int kQueryKeyBits = 30;         // bits of the query Hilbert keys (sorted as uint32)
constexpr int kBatchQueryMapShift = 30;   // batch query keys: (map id << 30) | 30-bit Hilbert index in the map's cell
struct QueryTuning {
    int layout;             // 0: lane per query with a shared-memory heap; 1: group buffers
    int queries_per_warp;   // group layout: 1, 2, 4 or 8 (32, 16, 8 or 4 lanes per query)
    int warps_per_block;
    int rounds_per_chunk;
    unsigned long long* stats;   // 8 traversal counters (group layout), nullptr = off
    const float4* qsorted = nullptr;   // query records in sorted order (pos.xyz | caller index, normal), or nullptr
};
int gather_queries(const uint32_t* order, const float4* qpos, const float4* qnrm, uint32_t nq, float4* out, cudaStream_t st);
int query_knn(const MapView& m, const QueryParams& p, const float4* qpos, const float4* qnrm,
              const uint32_t* order, uint32_t nq, const QueryOutputs& out, uint32_t* work_counter, uint32_t* fix_list,
              const QueryTuning& t, cudaStream_t st);
int query_bruteforce(const MapView& m, const QueryParams& p, const float4* qpos, const float4* qnrm,
                      uint32_t nq, const QueryOutputs& out, cudaStream_t st);
int query_smem_bytes_per_warp(uint32_t k);
double filter_norm_const(int filter, float cone_k);

int query_knn_batch(const MapView& m, const BatchQuery* bq, const BatchGeom* bg, uint32_t kmax, const float4* qpos,
                    const float4* qnrm, const uint32_t* order, const uint64_t* qkeys, uint32_t nq,
                    const QueryOutputs& out, uint32_t* work_counter, uint32_t* fix_list, const QueryTuning& t,
                    cudaStream_t st);

// pm_batch.cu
int batch_bounds_and_keys(const float4* pos, const float4* pw, const uint32_t* ph_off, uint32_t m, uint32_t n,
                          uint32_t* acc, BatchGeom* geom, MapHeader* hdr, uint64_t* keys, uint32_t* vals,
                          cudaStream_t st);
int batch_query_keys(const float4* qpos, const uint32_t* q_off, uint32_t m, uint32_t nq, const BatchGeom* geom,
                     uint64_t* keys, uint32_t* vals, cudaStream_t st);
int batch_roots(const uint32_t* ph_off, uint32_t m, uint32_t n, uint32_t leaf_size, const float4* pos,
                const Node* nodes, const BuildBuffers& bb, BatchGeom* geom, cudaStream_t st);
int map_id_bits(uint32_t m);
int batch_wide(uint32_t n, uint32_t m, const Node* nodes, const uint32_t* parent, MapHeader* hdr, uint32_t* rootmark,
               const WideBuffers& wb, BatchGeom* geom, cudaStream_t st);

// pm_compat.cu
int compat_node_estimates(const MapView& m, uint32_t max_slots, float rmax, uint32_t k, uint32_t iters, float* est,
                          cudaStream_t st);
int compat_query(const MapView& m, const float* est, const QueryParams& p, uint32_t iters, const float4* qpos,
                 const float4* qnrm, uint32_t nq, float* out_radius, const QueryOutputs& out, cudaStream_t st);

// pm_icut.cu: illumination cuts.  Per-slot arrays hold 2 (num_nodes + 1)
// entries (slot 2j + side of node j, slot 0 = root); pslot holds one entry
// per node.
struct IcutParams {
    bool use_leafs;
    uint32_t level_emin;
    uint32_t refine_iters;
    float accuracy;
};
struct IcutBuffers {
    uint32_t* pslot;             // node -> slot referencing it
    uint32_t* level;             // slot depth (root 0), kInvalid for empty slots
    uint2* range;                // slot photons [x, y) in tree order
    float4* center;              // box centre xyz, largest box side w
    float4* normal;              // normal xyz (zero: none)
    float4* est;                 // photon-sum estimate E~ (rgb)
    float4* exact;               // estimate at the centre (rgb, w = photons used)
    uint32_t* coarse;            // coarse cut marks
    uint32_t* fin;               // final cut marks
    uint32_t* work[2];           // work flags (refinement), mark scratch (coarse cut)
    unsigned long long* acc;     // level statistics: max bits [0..2], fixed sums [3..5], count [6]
    float4* ibox;                // per slot, 2 entries: influence box lo (w = 1: interpolation stops here), hi
};
int icut_prepare(const MapView& m, uint32_t num_nodes, const IcutBuffers& b, cudaStream_t st);
int icut_normals(const MapView& m, uint32_t nslots, const float4* caller, const IcutBuffers& b, cudaStream_t st);
int icut_coarse(const MapView& m, uint32_t nslots, const IcutParams& p, const IcutBuffers& b, cudaStream_t st);
int icut_final(const MapView& m, uint32_t nslots, const IcutParams& p, const IcutBuffers& b, cudaStream_t st);
int icut_interpolate(const MapView& m, const IcutBuffers& b, const float4* qpos, const float4* qnrm,
                     const uint32_t* order, uint32_t nq, float r2, float4* out, cudaStream_t st);

// pm_gather.cu
int gather_normals(const float4* hit_nrm, const float4* ray_dir, uint32_t n, float4* out_nrm, cudaStream_t st);
int gather_accumulate(const float4* est, const float4* hit_pos, const float4* ray_origin, const float4* influence,
                      const float4* clr_diffuse, const uint32_t* idx_shading, uint32_t n, float4* io_rad,
                      float* io_recip, cudaStream_t st);

int merge_ranks(const uint32_t* is_valid, uint32_t n, uint32_t* flags, uint32_t* rank, uint32_t* scan_scratch,
                uint32_t* total, cudaStream_t st);
int merge_scatter(const float4* pos, const float4* pw, const uint32_t* flags, const uint32_t* rank, uint32_t n,
                  float4* dst_pos, float4* dst_pow, cudaStream_t st);
int scale_rgb(float4* pw, uint32_t n, float scale, cudaStream_t st);

// pm_backward.cu
// Per-query record of the adjoint, 64 bytes: everything the per-photon pass
// needs about one query in one aligned load.
struct __align__(16) BwdQuery {
    double gx, gy, gz;        // dL/dE * norm per channel
    double G;                 // the k-th neighbour's r^2 path (0 unless k were found)
    double rinv;              // the filter's reciprocal: 1 / (k_c r) cone, 1 / r^2 Epanechnikov, 1 box;
                              // 0 = the query carries no gradient
    float qx, qy, qz;         // position
    float nx, ny, nz;         // normal
};
static_assert(sizeof(BwdQuery) == 64, "one 64-byte record per query");

struct BwdArgs {
    const float4* pos;        // tree order
    const float4* pow;
    const uint32_t* inv;      // caller index -> tree position
    const float4* qpos;       // all queries (indexed by global query id)
    const float4* qnrm;
    const float4* grad;       // dL/dE per query (rgb)
    const uint32_t* nbr;      // this chunk's neighbour rows (caller indices, sorted by (d^2, index))
    const uint32_t* count_in; // this chunk's counts, or nullptr (derived from the rows)
    uint32_t n, k;
    float r_max;
    int filter;
    float cone_k;
    uint32_t min_found;
    BwdQuery* qrec;           // per chunk query: the record the per-photon pass reads
    uint32_t* keys;           // sort path: one photon key per neighbour slot (set by backward_chunk)
    uint32_t* vals;           // pair values: grouped by photon (placement), or per slot (sort)
    uint32_t* cursor;         // per photon: pair count, then the next free slot of its segment
    uint64_t pair_cap;        // slots in vals
    const uint32_t* order;    // the chunk's queries in Hilbert order (chunk-local ids), or nullptr
};
struct BwdBuffers {
    uint32_t* vals[2];        // one slot per neighbour pair of a chunk ([1]: sort path only)
    uint32_t* keys[2];        // sort path only
    uint32_t* scratch;        // the scan of the per-photon counts, or the sort's
    uint32_t* seg_start;
    uint32_t* seg_end;
    uint32_t* long_list;      // photons whose segments a block sorts (n entries)
    uint32_t* long_count;
    double* acc;              // 6 doubles per photon, carried between chunks
};
// Mean pairs per photon above which a chunk groups its pairs by a stable
// radix sort instead of counts, atomic placement and segment sorts.
constexpr uint64_t kBwdPlaceMaxFanIn = 256;
inline bool bwd_sort_path(uint64_t pairs, uint32_t n) { return pairs > kBwdPlaceMaxFanIn * (uint64_t)n; }
size_t bwd_scratch_words(uint32_t n, uint64_t pairs, bool sort_path);
int backward_chunk(const BwdArgs& a, uint32_t q0, uint32_t nq_chunk, bool first, bool last, const BwdBuffers& b,
                   float4* grad_pow, float4* grad_pos, cudaStream_t st);

}  // namespace pm
