// pm_query.cu -- exact-kNN photon-map radiance estimate.
//
// Replaces dev_RangeSearch + kernel_PhotonGather (GPU/photon_knn.cu:113-235,
// 487-552) and the radius pipeline in front of it (KDTreePoint::
// ComputeQueryRadii, KDTreePoint.cpp:229-248).  Where the reference runs
// about three range searches per query (radius estimate, two histogram
// refinements, gather) with one thread and a local-memory stack per query,
// this kernel finds the exact k nearest photons in one pass:
//
//   * queries are processed in Hilbert order (k_query_order + the radix
//     sort; for the wide layout k_gather_queries then lays their 32-byte
//     records out in that order), and warps take chunks of consecutive
//     queries by guided self-scheduling (long chunks first, short ones last);
//   * each query starts from a radius bound given by the previous query of
//     its warp (triangle inequality: r_k(q) <= r_k(q') + |q - q'|), so most
//     searches start tight instead of at R;
//   * the default layout (PM_KBUF_WIDE, k_knn_group<32, *, *, true>) gives
//     each query a whole warp over the 32-wide tree: lane i tests child i,
//     passing leaves are scanned a photon per lane, candidates go to a
//     shared-memory buffer, and an exact selection keeps the k smallest
//     (d^2, caller index) keys; PM_KBUF_GROUP runs groups of lanes per query
//     over the binary tree, and PM_KBUF_HEAP (k_knn_tree) a lane per query
//     with a max-heap in shared memory, the warp traversing jointly;
//   * the cone / Epanechnikov / box filter and the 1/(pi r^2)
//     normalisation are fused into the epilogue; the weighted flux sum is
//     accumulated in 64-bit fixed point, so the result does not depend on
//     the order in which neighbours were found, and every layout gives the
//     same bits.
#include "pm_internal.h"

namespace pm {

constexpr uint32_t kFull = 0xffffffffu;

struct KnnArgs {
    const float4* pos;
    const float4* pow;
    const Node* nodes;
    MapHeader* hdr;
    const float4* qpos;
    const float4* qnrm;
    const uint32_t* order;   // sorted slot -> caller query index (nullptr = identity)
    uint32_t nq;
    uint32_t k;
    float r2max;
    float rmax;
    int filter;
    float cone_k;
    uint32_t min_found;
    float4* out_rad;
    uint32_t* out_nbr;
    float* out_r2;
    uint32_t* out_count;
    uint32_t* work_counter;
    uint32_t* fix_list;       // group kernel: sorted slots of queries whose estimate needs FP64 distances
    const uint32_t* fix_in;   // fix pass: the list it works through
    uint32_t* fix_count;
    const uint32_t* nq_dev;   // fix pass: query count read on the device
    uint32_t rounds_per_chunk;   // smallest chunk of the guided schedule, in rounds
    uint32_t cap;             // group kernel: candidate buffer entries per query
    uint32_t smem_per_warp;   // group kernel: shared bytes per warp
    unsigned long long* stats;   // optional traversal counters (kStat*), nullptr = off
    const float* scale_ptr;   // fixed-point scale of the flux sums (map header or batch map)
    const ChildSlot* root;    // slot the traversal starts from
    const ChildSlot* wchild;  // wide-tree child slots
    uint64_t nbr_off;         // batch: first neighbour slot of the map's rows
    uint32_t q_off;           // batch: first query of the map
    uint32_t ph_off;          // batch: first photon of the map (caller indices are batch-global)
    const uint64_t* qkeys;    // batch: sorted query keys, map id from bit kBatchQueryMapShift up
    const BatchGeom* bgeom;   // batch: per-map geometry (built)
    const BatchQuery* bq;     // batch: per-map query parameters
    double norm_c;            // the filter's normalisation constant (filter_norm_const)
    const float4* qsorted;    // query records in sorted order (pos.xyz | caller index, normal), or nullptr
    const ChildSlot* s_top;   // staged root children (shared memory) or nullptr
    uint32_t top_first;       // wchild index of the staged children
};

// Counters of the group kernel, accumulated when KnnArgs::stats is set.
enum { kStatQueries = 0, kStatNodes, kStatLeaves, kStatPhotons, kStatCandidates, kStatSelections, kStatRedo,
       kStatUnbounded, kStatCount };

// (d^2, position) keys; equal d^2 is resolved by the caller index stored in
// pos[].w, which keeps the order identical to (d^2, caller index).
__device__ __forceinline__ bool key_less(uint64_t a, uint64_t b, const float4* __restrict__ pos) {
    const uint32_t ah = (uint32_t)(a >> 32), bh = (uint32_t)(b >> 32);
    if (ah != bh) return ah < bh;
    if (a == b) return false;
    return __float_as_uint(pos[(uint32_t)a].w) < __float_as_uint(pos[(uint32_t)b].w);
}

// Max-heap helpers; element j of this lane lives at h[j * 32].
__device__ __forceinline__ void heap_push(uint64_t* h, uint32_t& hn, uint64_t v, const float4* pos) {
    uint32_t i = hn++;
    while (i > 0) {
        const uint32_t p = (i - 1) >> 1;
        const uint64_t pv = h[p * 32];
        if (!key_less(pv, v, pos)) break;
        h[i * 32] = pv;
        i = p;
    }
    h[i * 32] = v;
}

__device__ __forceinline__ void heap_sift_down(uint64_t* h, uint32_t n, uint64_t v, const float4* pos) {
    uint32_t i = 0;
    for (;;) {
        const uint32_t l = 2 * i + 1;
        if (l >= n) break;
        uint32_t c = l;
        uint64_t cv = h[l * 32];
        if (l + 1 < n) {
            const uint64_t rv = h[(l + 1) * 32];
            if (key_less(cv, rv, pos)) { c = l + 1; cv = rv; }
        }
        if (!key_less(v, cv, pos)) break;
        h[i * 32] = cv;
        i = c;
    }
    h[i * 32] = v;
}

// The estimate's arithmetic after the neighbour set is fixed runs in FP64,
// as the oracle's: weights from FP64 distances to the query, r^2 = FP64 d^2 of
// the k-th neighbour (or R^2).  Explicit roundings keep every kernel on the
// same bits.  The FP32 contract decides only the set, the front test and the
// reported r^2.
__device__ __forceinline__ double d2_64(double qx, double qy, double qz, const float4& p) {
    const double dx = __dsub_rn((double)p.x, qx), dy = __dsub_rn((double)p.y, qy), dz = __dsub_rn((double)p.z, qz);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Filter weight of one neighbour, relative error about 1e-7 however close
// the neighbour is to the edge of the ball: the cancelling difference
// delta = (k_c r)^2 - d^2 (cone) or r^2 - d^2 (Epanechnikov) is formed in FP64
// from FP64 distances, the rest in FP32.
//   cone:          w = 1 - d / (k_c r) = delta / (k_c r (k_c r + d))
//   Epanechnikov:  w = 1 - d^2 / r^2   = delta / r^2
struct Filter64 {
    int filter;
    double qx, qy, qz;
    double edge2;   // (k_c r)^2 (cone) or r^2 (Epanechnikov), FP64
    float edge;     // k_c r (cone)
    float inv;      // 1 / r^2 (Epanechnikov)
    __device__ __forceinline__ void init(int f, float cone_k, float x, float y, float z, double r2) {
        filter = f;
        qx = x; qy = y; qz = z;
        edge2 = 0.0; edge = 0.0f; inv = 0.0f;
        if (f == 1) {
            const double e = __dmul_rn((double)cone_k, __dsqrt_rn(r2));
            edge2 = __dmul_rn(__dmul_rn((double)cone_k, (double)cone_k), r2);   // exact r^2 for k_c = 1
            edge = __double2float_rn(e);
        } else if (f == 2) {
            edge2 = r2;
            inv = __double2float_rn(__drcp_rn(r2));
        }
    }
    __device__ __forceinline__ float weight(const float4& p) const {
        if (filter == 0) return 1.0f;
        const double d2 = d2_64(qx, qy, qz, p);
        const float delta = __double2float_rn(__dsub_rn(edge2, d2));
        if (filter == 2) return __fmul_rn(delta, inv);
        const float d = __fsqrt_rn(__double2float_rn(d2));
        return __fdiv_rn(delta, __fmul_rn(edge, __fadd_rn(edge, d)));
    }
};

// r^2 of the filter: FP64 d^2 of the k-th neighbour (tree position kth) when k
// were found, else R^2.
__device__ __forceinline__ double filter_r2(const float4* __restrict__ pos, bool full, uint32_t kth, float qx, float qy,
                                            float qz, float rmax) {
    if (!full) return __dmul_rn((double)rmax, (double)rmax);
    return d2_64(qx, qy, qz, __ldg(pos + kth));
}

__device__ __forceinline__ long long fixed_term(float w, float phi, float scale) {
    return __float2ll_rn(__fmul_rn(__fmul_rn(w, phi), scale));
}

// FP32 filter weights (the common path).  Their absolute error is below
// about 8e-7 (FP32 d^2 against FP64, the reciprocal square root, r), so a
// channel's relative error is below 8e-7 * sum(flux) / sum(w * flux) of that
// channel plus about 3e-7 from r^2: the FP32 path is kept when, in every
// channel, sum(w * flux) is at least sum(flux) / 6 (bound 5.1e-6), decided on
// the fixed-point sums (identical in every kernel); the query is re-evaluated
// with FP64 distances otherwise.
__device__ __forceinline__ float filter_inv32(int filter, float r2, float cone_k) {
    if (filter == 1) return __frcp_rn(__fmul_rn(cone_k, __fsqrt_rn(r2)));
    if (filter == 2) return __frcp_rn(r2);
    return 0.0f;
}

// The k-th neighbour's FP32 weight is 0 only up to that absolute error (its
// FP64 weight is exactly 1 - 1/k_c, 0 for k_c = 1); the per-channel FP64 test
// below sends every query where that matters to the FP64 path, which is exact
// on the edge.
__device__ __forceinline__ float filter_weight32(int filter, float d2, float inv) {
    if (filter == 1) {
        const float d = d2 > 0.0f ? __fmul_rn(d2, rsqrtf(d2)) : 0.0f;
        return fmaxf(__fsub_rn(1.0f, __fmul_rn(d, inv)), 0.0f);
    }
    if (filter == 2) return fmaxf(__fsub_rn(1.0f, __fmul_rn(d2, inv)), 0.0f);
    return 1.0f;
}

struct EstAcc {
    long long c0, c1, c2;   // weighted flux per channel, fixed point (scale s = fix_scale)
    uint32_t f0, f1, f2;    // |flux| per channel at s * 2^-29, each term rounded up
};

// One neighbour's terms from its loaded flux record w.
__device__ __forceinline__ void est_add32w(const KnnArgs& a, const float4& w, float d2, float inv, float nx, float ny,
                                           float nz, float scale, EstAcc& acc) {
    if (!front_rn(nx, ny, nz, __float_as_uint(w.w))) return;
    const float wt = filter_weight32(a.filter, d2, inv);
    acc.c0 += fixed_term(wt, w.x, scale);
    acc.c1 += fixed_term(wt, w.y, scale);
    acc.c2 += fixed_term(wt, w.z, scale);
    const float s32 = __fmul_rn(scale, 1.862645149230957e-09f);   // 2^-29
    acc.f0 += __float2uint_ru(__fmul_rn(fabsf(w.x), s32));
    acc.f1 += __float2uint_ru(__fmul_rn(fabsf(w.y), s32));
    acc.f2 += __float2uint_ru(__fmul_rn(fabsf(w.z), s32));
}

__device__ __forceinline__ void est_add32(const KnnArgs& a, uint32_t t, float d2, float inv, float nx, float ny,
                                          float nz, float scale, EstAcc& acc) {
    const float4 w = __ldg(a.pow + t);
    if (!front_rn(nx, ny, nz, __float_as_uint(w.w))) return;
    const float wt = filter_weight32(a.filter, d2, inv);
    acc.c0 += fixed_term(wt, w.x, scale);
    acc.c1 += fixed_term(wt, w.y, scale);
    acc.c2 += fixed_term(wt, w.z, scale);
    const float s32 = __fmul_rn(scale, 1.862645149230957e-09f);   // 2^-29
    acc.f0 += __float2uint_ru(__fmul_rn(fabsf(w.x), s32));
    acc.f1 += __float2uint_ru(__fmul_rn(fabsf(w.y), s32));
    acc.f2 += __float2uint_ru(__fmul_rn(fabsf(w.z), s32));
}

__device__ __forceinline__ void est_add64(const KnnArgs& a, uint32_t t, const Filter64& flt, float nx, float ny,
                                          float nz, float scale, EstAcc& acc) {
    const float4 w = __ldg(a.pow + t);
    if (!front_rn(nx, ny, nz, __float_as_uint(w.w))) return;
    const float wt = flt.weight(__ldg(a.pos + t));
    acc.c0 += fixed_term(wt, w.x, scale);
    acc.c1 += fixed_term(wt, w.y, scale);
    acc.c2 += fixed_term(wt, w.z, scale);
}

// Per channel: the FP32 weights' absolute error becomes a relative error of
// that channel's estimate scaled by its sum(flux) / sum(w * flux), so every
// channel must pass on its own (a channel whose flux sits in low-weight
// neighbours, e.g. the k-th at weight zero, would otherwise slip through).
// The unweighted sums are kept in 32 bits at 2^24 / max flux with every term
// rounded up, which can only send more queries to FP64.  The comparison
// 6 sum(w flux) < sum(flux) is exact in 64-bit integers: the weighted sums are
// below 2^60 (6 times that below 2^63), the unweighted ones below 2^31.
__device__ __forceinline__ bool est_needs_fp64(int filter, const EstAcc& acc) {
    if (filter == 0) return false;
    return 6ll * acc.c0 < (long long)((uint64_t)acc.f0 << 29) || 6ll * acc.c1 < (long long)((uint64_t)acc.f1 << 29) ||
           6ll * acc.c2 < (long long)((uint64_t)acc.f2 << 29);
}

// The estimate from the fixed-point sums: c / (r^2 scale) per unit of sum, c
// the filter's normalisation constant (filter_norm_const, one FP64 division
// per query).
__device__ __forceinline__ float4 est_result(const EstAcc& acc, double r2, float scale, uint32_t n, double norm_c) {
    float4 rad = make_float4(0.0f, 0.0f, 0.0f, (float)n);
    if (scale > 0.0f) {
        const double f = norm_c / __dmul_rn(r2, (double)scale);
        rad.x = __double2float_rn((double)acc.c0 * f);
        rad.y = __double2float_rn((double)acc.c1 * f);
        rad.z = __double2float_rn((double)acc.c2 * f);
    }
    return rad;
}


// The FP64 re-evaluation of one query (rare path).  Returns r^2 in FP64.
__device__ __forceinline__ double est_fp64_heap(const KnnArgs& a, const uint64_t* h, uint32_t stride, uint32_t hn,
                                             bool full, uint32_t kth, float qx, float qy, float qz, float nx, float ny,
                                             float nz, EstAcc& acc) {
    const double r2d = filter_r2(a.pos, full, kth, qx, qy, qz, a.rmax);
    const float scale = *a.scale_ptr;
    Filter64 flt;
    flt.init(a.filter, a.cone_k, qx, qy, qz, r2d);
    acc = EstAcc{0, 0, 0, 0, 0, 0};
    for (uint32_t j = 0; j < hn; ++j) est_add64(a, (uint32_t)h[j * stride], flt, nx, ny, nz, scale, acc);
    return r2d;
}

// Epilogue for one lane: fixed-point filtered flux sum over the heap, optional
// sorted neighbour list.  Shared by the tree and the brute-force kernels.
// stride: distance between consecutive heap elements of this lane.
__device__ void finish_query(const KnnArgs& a, uint64_t* h, uint32_t stride, uint32_t hn, uint32_t qo, float qx,
                             float qy, float qz, float nx, float ny, float nz) {
    const uint32_t k = a.k;
    const float r2 = (hn == k) ? __uint_as_float((uint32_t)(h[0] >> 32)) : a.r2max;
    const uint32_t kth = (uint32_t)h[0];   // tree position of the k-th (heap top) when hn == k
    if (a.out_nbr) {   // heapsort in place -> ascending (d^2, index)
        for (uint32_t end = hn; end > 1; --end) {
            const uint64_t top = h[0];
            const uint64_t last = h[(end - 1) * stride];
            h[(end - 1) * stride] = top;
            // sift `last` down within [0, end - 1)
            uint32_t i = 0;
            const uint32_t n = end - 1;
            for (;;) {
                const uint32_t l = 2 * i + 1;
                if (l >= n) break;
                uint32_t c = l;
                uint64_t cv = h[l * stride];
                if (l + 1 < n) {
                    const uint64_t rv = h[(l + 1) * stride];
                    if (key_less(cv, rv, a.pos)) { c = l + 1; cv = rv; }
                }
                if (!key_less(last, cv, a.pos)) break;
                h[i * stride] = cv;
                i = c;
            }
            h[i * stride] = last;
        }
        uint32_t* row = a.out_nbr + (size_t)qo * k;
        for (uint32_t j = 0; j < k; ++j)
            row[j] = (j < hn) ? __float_as_uint(a.pos[(uint32_t)h[j * stride]].w) : kInvalid;
    }
    float4 rad = make_float4(0.0f, 0.0f, 0.0f, (float)hn);
    if (hn > 0 && hn >= a.min_found && r2 > 0.0f) {
        const float scale = *a.scale_ptr;
        const float inv = filter_inv32(a.filter, r2, a.cone_k);
        EstAcc acc = {0, 0, 0, 0, 0, 0};
        for (uint32_t j = 0; j < hn; ++j) {
            const uint64_t key = h[j * stride];
            est_add32(a, (uint32_t)key, __uint_as_float((uint32_t)(key >> 32)), inv, nx, ny, nz, scale, acc);
        }
        double r2d = (double)r2;
        if (est_needs_fp64(a.filter, acc)) r2d = est_fp64_heap(a, h, stride, hn, hn == k, kth, qx, qy, qz, nx, ny, nz, acc);
        rad = est_result(acc, r2d, scale, hn, a.norm_c);
    }
    a.out_rad[qo] = rad;
    if (a.out_r2) a.out_r2[qo] = r2;
    if (a.out_count) a.out_count[qo] = hn;
}

__device__ __forceinline__ void load_slot(const Node* nodes, uint32_t node, uint32_t side, float* lo, float* hi,
                                          uint32_t& ref, uint32_t& cnt) {
    const float4* p = reinterpret_cast<const float4*>(&nodes[node].c[side]);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    lo[0] = a.x; lo[1] = a.y; lo[2] = a.z; hi[0] = a.w;
    hi[1] = b.x; hi[2] = b.y; ref = __float_as_uint(b.z); cnt = __float_as_uint(b.w);
}

__device__ __forceinline__ void load_root(const ChildSlot* slot, float* lo, float* hi, uint32_t& ref, uint32_t& cnt) {
    const float4* p = reinterpret_cast<const float4*>(slot);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    lo[0] = a.x; lo[1] = a.y; lo[2] = a.z; hi[0] = a.w;
    hi[1] = b.x; hi[2] = b.y; ref = __float_as_uint(b.z); cnt = __float_as_uint(b.w);
}

// Guided self-scheduling (Polychronopoulos & Kuck, 1987) of the sorted
// queries, in rounds (a round = the queries one warp takes at once): warps
// take chunk numbers from one atomic counter; group g holds P chunks (P = the
// grid's warps) of s_g = max(rmin, rem_g / 2P + 1) rounds each, rem_g the
// rounds left before the group.  Early chunks are long, so fewer queries
// start without the radius bound of their predecessor (every chunk's first
// query does); the last chunks are rmin rounds, so the launch's tail stays
// short.  Against fixed 32-round chunks: 65k -> 31k chunks on 2.07M queries
// and 7.62 -> 7.29 ms for the query kernel.  rmax caps a chunk where query
// costs differ widely (a batch of maps with different k and sizes: uncapped,
// one chunk of costly queries outlasts the rest of the launch).  Returns
// false past the end.
__device__ __forceinline__ bool guided_chunk(uint32_t c, uint32_t total, uint32_t P, uint32_t rmin, uint32_t rmax,
                                             uint32_t& begin, uint32_t& len) {
    uint32_t base = 0;
    for (;;) {
        if (base >= total) return false;
        const uint32_t s = max(rmin, min(rmax, (total - base) / (2u * P) + 1u));
        if (c < P) {
            const uint64_t b = (uint64_t)base + (uint64_t)c * s;
            if (b >= total) return false;
            begin = (uint32_t)b;
            len = min(s, total - (uint32_t)b);
            return true;
        }
        c -= P;
        const uint64_t nb = (uint64_t)base + (uint64_t)P * s;
        base = nb >= total ? total : (uint32_t)nb;
    }
}

// One warp = 32 queries (one per lane) traversing together.
__global__ void __launch_bounds__(256) k_knn_tree(KnnArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = lane_id();
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t k = a.k;
    const size_t per_warp = (size_t)32 * k * sizeof(uint64_t) + kStackDepth * sizeof(uint32_t);
    unsigned char* wbase = smem + per_warp * warp;
    uint64_t* heap = reinterpret_cast<uint64_t*>(wbase) + lane;
    uint32_t* stack = reinterpret_cast<uint32_t*>(wbase + (size_t)32 * k * sizeof(uint64_t));
    const float r2max = a.r2max;
    const uint32_t total_rounds = (a.nq + 31u) / 32u;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);

    for (;;) {
        uint32_t chunk = 0;
        if (lane == 0) chunk = atomicAdd(a.work_counter, 1u);
        chunk = __shfl_sync(kFull, chunk, 0);
        uint32_t rbegin = 0, rlen = 0;
        if (!guided_chunk(chunk, total_rounds, nwarps, a.rounds_per_chunk, 0xffffffffu, rbegin, rlen)) break;
        // previous round's result of this lane (for the radius bound)
        float pqx = 0.f, pqy = 0.f, pqz = 0.f, pr = 0.f;
        bool pvalid = false;
        for (uint32_t round = 0; round < rlen; ++round) {
            const uint32_t slot_q = (rbegin + round) * 32 + lane;
            const bool inrange = slot_q < a.nq;
            if (!__any_sync(kFull, inrange)) break;
            uint32_t qo = 0;
            float qx = 0.f, qy = 0.f, qz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
            bool active = false;
            if (inrange) {
                qo = a.order ? a.order[slot_q] : slot_q;
                const float4 q = a.qpos[qo];
                const float4 nn = a.qnrm[qo];
                qx = q.x; qy = q.y; qz = q.z; nx = nn.x; ny = nn.y; nz = nn.z;
                active = isfinite(qx) && isfinite(qy) && isfinite(qz);
                if (!active) atomicOr(&a.hdr->errors, kErrQueryNonFinite);
            }
            // radius bound from the previous round's 32 queries
            float tau0 = r2max;
#pragma unroll 4
            for (int s = 0; s < 32; ++s) {
                const float sx = __shfl_sync(kFull, pqx, s), sy = __shfl_sync(kFull, pqy, s);
                const float sz = __shfl_sync(kFull, pqz, s), sr = __shfl_sync(kFull, pr, s);
                const bool sv = __shfl_sync(kFull, pvalid, s);
                if (sv) {
                    const float dq = __fsqrt_rn(d2_rn(qx, qy, qz, sx, sy, sz));
                    const float b = __fmul_rn(__fadd_rn(sr, dq), 1.000244140625f);
                    tau0 = fminf(tau0, __fmul_rn(__fmul_rn(b, b), 1.000244140625f));
                }
            }
            uint32_t hn = 0;
            bool full = false, todo = active;
            while (__any_sync(kFull, todo)) {
                // (re)start the search of the lanes in `todo`
                const bool live = todo;
                if (live) { hn = 0; full = false; }
                uint64_t top = 0;
                float tauf = 0.0f;
                int sp = 0;
                // current slot = the root slot of the super-root
                float lo[3], hi[3];
                uint32_t ref, cnt;
                load_slot(a.nodes, 0, 0, lo, hi, ref, cnt);
                bool have = true;
                {
                    const float lb = box_lb(qx, qy, qz, lo, hi);
                    have = __any_sync(kFull, live && lb < tau0) && ref != kInvalid;
                }
                for (;;) {
                    if (have) {
                        if (cnt > 0) {
                            // leaf: 32 photons at a time, a coalesced load broadcast photon by photon
                            for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
                                float4 mine = make_float4(0.f, 0.f, 0.f, 0.f);
                                if (c0 + lane < cnt) mine = __ldg(a.pos + ref + c0 + lane);
                                const uint32_t cn = min(cnt - c0, 32u);
                                for (uint32_t j = 0; j < cn; ++j) {
                                    const float px = __shfl_sync(kFull, mine.x, j);
                                    const float py = __shfl_sync(kFull, mine.y, j);
                                    const float pz = __shfl_sync(kFull, mine.z, j);
                                    if (!live) continue;
                                    const float d2 = d2_rn(qx, qy, qz, px, py, pz);
                                    const uint64_t key = ((uint64_t)__float_as_uint(d2) << 32) | (ref + c0 + j);
                                    if (!full) {
                                        if (d2 < tau0) {
                                            heap_push(heap, hn, key, a.pos);
                                            if (hn == k) { full = true; top = heap[0]; tauf = __uint_as_float((uint32_t)(top >> 32)); }
                                        }
                                    } else if (key_less(key, top, a.pos)) {
                                        heap_sift_down(heap, k, key, a.pos);
                                        top = heap[0];
                                        tauf = __uint_as_float((uint32_t)(top >> 32));
                                    }
                                }
                            }
                            have = false;
                        } else {
                            float l0[3], h0[3], l1[3], h1[3];
                            uint32_t r0, c0, r1, c1;
                            load_slot(a.nodes, ref, 0, l0, h0, r0, c0);
                            load_slot(a.nodes, ref, 1, l1, h1, r1, c1);
                            const float lb0 = box_lb(qx, qy, qz, l0, h0);
                            const float lb1 = box_lb(qx, qy, qz, l1, h1);
                            const bool p0 = live && (full ? lb0 <= tauf : lb0 < tau0);
                            const bool p1 = live && (full ? lb1 <= tauf : lb1 < tau0);
                            const uint32_t b0 = __ballot_sync(kFull, p0), b1 = __ballot_sync(kFull, p1);
                            const bool w0 = b0 != 0 && r0 != kInvalid, w1 = b1 != 0 && r1 != kInvalid;
                            if (w0 && w1) {
                                const uint32_t votes = __ballot_sync(kFull, (p0 || p1) && lb1 < lb0);
                                const uint32_t voters = b0 | b1;
                                const int near = (2 * __popc(votes) > __popc(voters)) ? 1 : 0;
                                if (sp >= kStackDepth) {
                                    if (lane == 0) atomicOr(&a.hdr->errors, kErrStack);
                                } else {
                                    if (lane == 0) stack[sp] = (ref << 1) | (uint32_t)(1 - near);
                                    ++sp;
                                }
                                if (near) { lo[0] = l1[0]; lo[1] = l1[1]; lo[2] = l1[2]; hi[0] = h1[0]; hi[1] = h1[1]; hi[2] = h1[2]; ref = r1; cnt = c1; }
                                else { lo[0] = l0[0]; lo[1] = l0[1]; lo[2] = l0[2]; hi[0] = h0[0]; hi[1] = h0[1]; hi[2] = h0[2]; ref = r0; cnt = c0; }
                            } else if (w0) {
                                ref = r0; cnt = c0;
                            } else if (w1) {
                                ref = r1; cnt = c1;
                            } else {
                                have = false;
                            }
                        }
                        continue;
                    }
                    // pop until a slot passes some lane's current threshold
                    bool found = false;
                    while (sp > 0) {
                        --sp;
                        __syncwarp();
                        const uint32_t e = stack[sp];
                        load_slot(a.nodes, e >> 1, e & 1u, lo, hi, ref, cnt);
                        const float lb = box_lb(qx, qy, qz, lo, hi);
                        const bool p = live && (full ? lb <= tauf : lb < tau0);
                        if (__any_sync(kFull, p)) { found = true; break; }
                    }
                    if (!found) break;
                    have = true;
                }
                // a bound that admitted fewer than k photons was too tight: redo with R
                todo = live && !full && tau0 < r2max;
                if (todo) tau0 = r2max;
                __syncwarp();
            }
            // k-th distance of this lane, read before the epilogue reorders the heap
            const float rk2 = (active && full) ? __uint_as_float((uint32_t)(heap[0] >> 32)) : 0.0f;
            if (inrange) {
                if (active) {
                    finish_query(a, heap, 32, hn, qo, qx, qy, qz, nx, ny, nz);
                } else {
                    a.out_rad[qo] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (a.out_r2) a.out_r2[qo] = r2max;
                    if (a.out_count) a.out_count[qo] = 0;
                    if (a.out_nbr)
                        for (uint32_t j = 0; j < k; ++j) a.out_nbr[(size_t)qo * k + j] = kInvalid;
                }
            }
            pqx = qx; pqy = qy; pqz = qz;
            pvalid = active && full;
            pr = pvalid ? __fsqrt_rn(rk2) : 0.0f;
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------------
// Group kernel: G lanes per query, 32 / G queries per warp.
//
// The warp traverses the tree jointly for its 32 / G queries (a child is
// visited when any query's box bound passes its threshold).  At a leaf the G
// lanes of a group split the leaf's photons; accepted candidates are
// appended to the group's buffer in shared memory with one ballot per step
// (no per-candidate dependent chains).  When the buffer fills, an exact
// selection keeps the k smallest (d^2, caller index) keys and tightens the
// threshold (group_select: one 8-bit histogram round finds the boundary
// bucket, whose few keys are ranked exactly).

template <int G>
struct GroupCtx {
    static constexpr int QW = 32 / G;
    uint32_t s;       // sub-lane 0..G-1
    uint32_t gbase;   // first lane of the group
    uint32_t gmask;   // lanes of the group
};

template <int G>
__device__ __forceinline__ uint32_t gmax_u32(uint32_t v, uint32_t gmask) {
    return __reduce_max_sync(gmask, v);   // one warp reduction instruction (measured 7.92 -> 7.85 ms)
}
template <int G>
__device__ __forceinline__ uint32_t gsum_u32(uint32_t v, uint32_t gmask) {
#pragma unroll
    for (int o = G / 2; o; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}
template <int G>
__device__ __forceinline__ long long gsum_i64(long long v, uint32_t gmask) {
#pragma unroll
    for (int o = G / 2; o; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
    return v;
}
template <int G>
__device__ __forceinline__ uint64_t gmin_u64(uint64_t v, uint32_t gmask) {
#pragma unroll
    for (int o = G / 2; o; o >>= 1) {
        const uint64_t w = __shfl_xor_sync(gmask, v, o);
        v = w < v ? w : v;
    }
    return v;
}
// exclusive prefix over the group's lanes
template <int G>
__device__ __forceinline__ uint32_t gexscan_u32(uint32_t v, uint32_t s, uint32_t gmask) {
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        const uint32_t y = __shfl_up_sync(gmask, x, o, G);
        if (s >= (uint32_t)o) x += y;
    }
    return x - v;
}

// A query started without a radius bound when its first search used R.
__device__ __forceinline__ bool pvalid_any_bound(float tau0, float r2max, uint32_t redo) {
    return redo == 0 && tau0 < r2max;
}

__device__ __forceinline__ uint32_t q16(uint32_t d2bits, float scale) {
    const float t = __fmul_rn(__uint_as_float(d2bits), scale);
    return t >= 65535.0f ? 65535u : (uint32_t)t;
}

__device__ __forceinline__ uint64_t exact_key(uint64_t e, const float4* __restrict__ pos) {
    return (e & 0xffffffff00000000ull) | __float_as_uint(pos[(uint32_t)e].w);
}

// One histogram round: finds the bucket (8-bit digit) holding the kk-th entry
// among entries whose quantised key has `prefix` in the bits above `shift`
// (prefix_shift = 16 means every entry).  Returns digit; kk is reduced by the
// count of entries in lower buckets.
template <int G>
__device__ uint32_t hist_round(const uint64_t* buf, uint32_t n, float scale, int shift, uint32_t prefix,
                               bool use_prefix, uint32_t& kk, uint32_t* hist, uint32_t s, uint32_t gmask) {
    constexpr int BPL = 256 / G;   // buckets per lane
    uint4* own = reinterpret_cast<uint4*>(hist + s * BPL);   // this lane's buckets, 16-byte aligned
#pragma unroll
    for (int i = 0; i < BPL / 4; ++i) own[i] = make_uint4(0u, 0u, 0u, 0u);
    __syncwarp(gmask);
    for (uint32_t e = s; e < n; e += G) {
        const uint32_t q = q16(reinterpret_cast<const uint32_t*>(buf)[2 * e + 1], scale);   // the d^2 word
        if (!use_prefix || (q >> 8) == prefix) atomicAdd(&hist[(q >> shift) & 255u], 1u);
    }
    __syncwarp(gmask);
    uint32_t local = 0, digit = 0, below = 0;
    bool mine;
    if constexpr (BPL <= 8) {   // one warp per query: the lane's 8 buckets stay in registers
        uint32_t h[BPL];
#pragma unroll
        for (int i = 0; i < BPL / 4; ++i) {
            const uint4 v = own[i];
            h[4 * i] = v.x; h[4 * i + 1] = v.y; h[4 * i + 2] = v.z; h[4 * i + 3] = v.w;
        }
#pragma unroll
        for (int i = 0; i < BPL; ++i) local += h[i];
        const uint32_t base = gexscan_u32<G>(local, s, gmask);
        mine = base < kk && kk <= base + local;
        uint32_t run = base;
        bool found = false;
#pragma unroll
        for (int i = 0; i < BPL; ++i) {
            if (mine && !found && run + h[i] >= kk) { digit = s * BPL + i; below = run; found = true; }
            run += h[i];
        }
    } else {
#pragma unroll
        for (int i = 0; i < BPL; ++i) local += hist[s * BPL + i];
        const uint32_t base = gexscan_u32<G>(local, s, gmask);
        mine = base < kk && kk <= base + local;
        if (mine) {
            uint32_t run = base;
            for (int i = 0; i < BPL; ++i) {
                const uint32_t hv = hist[s * BPL + i];
                if (run + hv >= kk) { digit = s * BPL + i; below = run; break; }
                run += hv;
            }
        }
    }
    const uint32_t who = __ffs(__ballot_sync(gmask, mine)) - 1;
    digit = __shfl_sync(gmask, digit, who);
    below = __shfl_sync(gmask, below, who);
    kk -= below;
    __syncwarp(gmask);
    return digit;
}

// General selection (any distribution of keys): two 8-bit histogram rounds
// on d^2 quantised to 16 bits, then an exact pass over the boundary bucket.
template <int G>
__device__ uint64_t group_select_general(uint64_t* buf, uint32_t& n, uint32_t kk, uint32_t* hist,
                                 const float4* __restrict__ pos, uint32_t s, uint32_t gmask, uint32_t lt) {
    uint32_t mx = 0;
    for (uint32_t e = s; e < n; e += G) mx = max(mx, (uint32_t)(buf[e] >> 32));
    mx = gmax_u32<G>(mx, gmask);
    const float dmax = __uint_as_float(mx);
    const float scale = dmax > 0.0f ? __fdiv_rn(65535.0f, dmax) : 0.0f;
    uint32_t need = kk;
    const uint32_t b1 = hist_round<G>(buf, n, scale, 8, 0, false, need, hist, s, gmask);
    const uint32_t b2 = hist_round<G>(buf, n, scale, 0, b1, true, need, hist, s, gmask);
    const uint32_t K16 = (b1 << 8) | b2;
    // exact pass over the boundary bucket: `need` smallest exact keys
    uint64_t T = 0;
    bool first = true;
    for (uint32_t t = 0; t < need; ++t) {
        uint64_t best = ~0ull;
        for (uint32_t e = s; e < n; e += G) {
            const uint64_t v = buf[e];
            if (q16((uint32_t)(v >> 32), scale) != K16) continue;
            const uint64_t x = exact_key(v, pos);
            if ((first || x > T) && x < best) best = x;
        }
        T = gmin_u64<G>(best, gmask);
        first = false;
    }
    // compact in place, keeping order of appearance
    uint32_t out = 0;
    for (uint32_t base = 0; base < n; base += G) {
        const uint32_t e = base + s;
        uint64_t v = 0;
        bool keep = false;
        if (e < n) {
            v = buf[e];
            const uint32_t q = q16((uint32_t)(v >> 32), scale);
            keep = q < K16 || (q == K16 && exact_key(v, pos) <= T);
        }
        const uint32_t bal = __ballot_sync(gmask, keep);
        __syncwarp(gmask);
        if (keep) buf[out + __popc(bal & lt)] = v;
        out += __popc(bal);
        __syncwarp(gmask);
    }
    n = out;
    return T;
}

// Sorts one 64-bit key per lane of a group of G lanes (bitonic network).
template <int G>
__device__ __forceinline__ uint64_t gsort_bitonic(uint64_t v, uint32_t s, uint32_t gmask) {
#pragma unroll
    for (int size = 2; size <= G; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const uint64_t o = __shfl_xor_sync(gmask, v, stride);
            const bool up = (s & (uint32_t)size) == 0;
            const bool lower = (s & (uint32_t)stride) == 0;
            v = (lower == up) ? (o < v ? o : v) : (o > v ? o : v);
        }
    }
    return v;
}

// Keeps exactly kk entries of buf[0, n): the kk smallest (d^2, caller index),
// in order of appearance; returns the d^2 bits of the kk-th in the high word.
// One 8-bit histogram round on d^2 quantised to [0, 255] finds the boundary
// bucket B.  On a surface d^2 is close to uniform, so B holds one or two
// entries: when all of B is kept no caller index is read at all, and when
// part of it is, its entries (at most G) are ranked by one bitonic sort of
// their exact keys.  Anything else takes group_select_general.
// Out of line: called about once per query, and inlined at both call sites it
// crowds the hot loop's instructions.
template <int G>
__device__ __noinline__ uint64_t group_select(uint64_t* buf, uint32_t& n, uint32_t kk, uint32_t* hist,
                                              const float4* __restrict__ pos, uint32_t s, uint32_t gmask, uint32_t lt,
                                              float bound) {
    float dmax = bound;   // every entry's d^2 is at most the acceptance threshold
    if (!(dmax > 0.0f) || !(dmax < INFINITY)) {
        uint32_t mx = 0;
        for (uint32_t e = s; e < n; e += G) mx = max(mx, (uint32_t)(buf[e] >> 32));
        mx = gmax_u32<G>(mx, gmask);
        dmax = __uint_as_float(mx);
    }
    if (!(dmax > 0.0f)) return group_select_general<G>(buf, n, kk, hist, pos, s, gmask, lt);
    const float scale = __fdiv_rn(255.0f, dmax);   // q in [0, 255], monotone in d^2
    uint32_t need = kk;
    const uint32_t B = hist_round<G>(buf, n, scale, 0, 0, false, need, hist, s, gmask);
    const uint32_t nb = hist[B];
    __syncwarp(gmask);
    const bool all_b = need == nb;
    if (!all_b && nb > (uint32_t)G) return group_select_general<G>(buf, n, kk, hist, pos, s, gmask, lt);
    uint64_t T = ~0ull;
    if (!all_b) {   // rank the boundary bucket's exact keys
        uint64_t* bl = reinterpret_cast<uint64_t*>(hist);   // 128 slots of this group's histogram space
        uint32_t got = 0;
        for (uint32_t base = 0; base < n; base += G) {
            const uint32_t e = base + s;
            const bool in_b = e < n && q16((uint32_t)(buf[e] >> 32), scale) == B;
            const uint32_t bal = __ballot_sync(gmask, in_b);
            if (in_b) bl[got + __popc(bal & lt)] = buf[e];
            got += __popc(bal);
        }
        __syncwarp(gmask);
        const uint64_t x = s < nb ? exact_key(bl[s], pos) : ~0ull;
        const uint64_t sorted = gsort_bitonic<G>(x, s, gmask);
        T = __shfl_sync(gmask, sorted, (int)(__ffs(gmask) - 1u + need - 1u));   // the need-th of B
        __syncwarp(gmask);
    }
    uint32_t out = 0, kmax = 0;
    for (uint32_t base = 0; base < n; base += G) {
        const uint32_t e = base + s;
        uint64_t v = 0;
        bool keep = false;
        if (e < n) {
            v = buf[e];
            const uint32_t q = q16((uint32_t)(v >> 32), scale);
            keep = q < B || (q == B && (all_b || exact_key(v, pos) <= T));
        }
        const uint32_t bal = __ballot_sync(gmask, keep);
        __syncwarp(gmask);   // this round's reads before its writes (in place, never ahead of the reads)
        if (keep) {
            buf[out + __popc(bal & lt)] = v;
            kmax = max(kmax, (uint32_t)(v >> 32));
        }
        out += __popc(bal);
    }
    __syncwarp(gmask);
    n = out;
    return (uint64_t)gmax_u32<G>(kmax, gmask) << 32;
}

// Final selection and outputs for one query held by a group of G lanes:
// keeps the k nearest, writes radiance / r^2 / count / sorted neighbours and
// returns the r^2 used by the filter.
// Tree position of the k-th neighbour (the largest exact key (d^2, caller
// index)) of a full group buffer; caller indices are read only for entries
// that share the largest d^2.
template <int G>
__device__ uint32_t group_kth(const KnnArgs& a, const uint64_t* buf, uint32_t n, uint32_t s, uint32_t gmask) {
    uint32_t mx = 0;
    for (uint32_t e = s; e < n; e += G) mx = max(mx, (uint32_t)(buf[e] >> 32));
    mx = gmax_u32<G>(mx, gmask);
    uint64_t best = 0;   // exact key + 1; 0 = no entry with the largest d^2 in this lane
    uint32_t bpos = 0;
    for (uint32_t e = s; e < n; e += G) {
        const uint64_t v = buf[e];
        if ((uint32_t)(v >> 32) != mx) continue;
        const uint64_t x = exact_key(v, a.pos) + 1ull;
        if (x > best) { best = x; bpos = (uint32_t)v; }
    }
#pragma unroll
    for (int o = G / 2; o; o >>= 1) {
        const uint64_t ob = __shfl_xor_sync(gmask, best, o);
        const uint32_t op = __shfl_xor_sync(gmask, bpos, o);
        if (ob > best) { best = ob; bpos = op; }
    }
    return bpos;
}

template <int G>
__device__ __forceinline__ double est_fp64_group(const KnnArgs& a, const uint64_t* buf, uint32_t n, uint32_t s,
                                              uint32_t gmask, float qx, float qy, float qz, float nx, float ny,
                                              float nz, EstAcc& acc) {
    const bool full = n == a.k;
    const uint32_t kth = full ? group_kth<G>(a, buf, n, s, gmask) : 0u;
    const double r2d = filter_r2(a.pos, full, kth, qx, qy, qz, a.rmax);
    const float scale = *a.scale_ptr;
    Filter64 flt;
    flt.init(a.filter, a.cone_k, qx, qy, qz, r2d);
    acc = EstAcc{0, 0, 0, 0, 0, 0};
    for (uint32_t e = s; e < n; e += G) est_add64(a, (uint32_t)buf[e], flt, nx, ny, nz, scale, acc);
    acc.c0 = gsum_i64<G>(acc.c0, gmask);
    acc.c1 = gsum_i64<G>(acc.c1, gmask);
    acc.c2 = gsum_i64<G>(acc.c2, gmask);
    return r2d;
}

// The sorted neighbour row of one query: the n kept keys, made exact
// ((d^2, caller index), unique), padded to a power of two and bitonic-sorted
// in place in the group's buffer (capacity >= that power of two).  Out of
// line and with scalar arguments: only list-producing calls reach it, and
// keeping it out of the hot instance measured 7.85 -> 7.61 ms together with
// the statistics compiled out of the wide instances.
template <int G>
__device__ __noinline__ void write_neighbours(uint64_t* buf, uint32_t n, uint32_t s, uint32_t gmask,
                                              const float4* __restrict__ pos, uint32_t* row, uint32_t k,
                                              uint32_t ph_off) {
    uint32_t N = 1;
    while (N < n) N <<= 1;
    for (uint32_t e = s; e < N; e += G) buf[e] = e < n ? exact_key(buf[e], pos) : ~0ull;
    __syncwarp(gmask);
    for (uint32_t size = 2; size <= N; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = s; i < N / 2; i += G) {
                const uint32_t lo = ((i & ~(stride - 1u)) << 1) | (i & (stride - 1u)), hi = lo + stride;
                const uint64_t x = buf[lo], y = buf[hi];
                const bool up = (lo & size) == 0;
                if ((x > y) == up) { buf[lo] = y; buf[hi] = x; }
            }
            __syncwarp(gmask);
        }
    }
    for (uint32_t e = s; e < n; e += G) row[e] = (uint32_t)buf[e] - ph_off;
    for (uint32_t j = n + s; j < k; j += G) row[j] = kInvalid;
    __syncwarp(gmask);
}

template <int G, bool kFix>
__device__ float group_finish(const KnnArgs& a, uint64_t* buf, uint32_t& n, uint32_t* hist, float thr, uint32_t s,
                              uint32_t gmask, uint32_t lt, uint32_t qo, uint32_t slot, float qx, float qy, float qz,
                              float nx, float ny, float nz) {
    const uint32_t k = a.k;
    float rk2 = a.r2max;
    if (n > k) {   // the selection returns the largest kept d^2, the k-th neighbour's
        rk2 = __uint_as_float((uint32_t)(group_select<G>(buf, n, k, hist, a.pos, s, gmask, lt, thr) >> 32));
    } else if (n == k) {
        uint32_t mx = 0;
        for (uint32_t e = s; e < n; e += G) mx = max(mx, reinterpret_cast<const uint32_t*>(buf)[2 * e + 1]);
        rk2 = __uint_as_float(gmax_u32<G>(mx, gmask));
    }
    const float r2 = rk2;
    float4 rad = make_float4(0.f, 0.f, 0.f, (float)n);
    if (n > 0 && n >= a.min_found && r2 > 0.0f) {
        const float scale = *a.scale_ptr;
        const float inv = filter_inv32(a.filter, r2, a.cone_k);
        EstAcc acc = {0, 0, 0, 0, 0, 0};
        // two neighbours per step, both flux records requested before either is
        // used (measured 8.34 -> 8.07 ms; four at once spills)
        for (uint32_t e = s; e < n; e += 2 * G) {
            const uint64_t k0 = buf[e];
            const bool has1 = e + G < n;
            const uint64_t k1 = has1 ? buf[e + G] : k0;
            const float4 w0 = __ldg(a.pow + (uint32_t)k0);
            const float4 w1 = __ldg(a.pow + (uint32_t)k1);
            est_add32w(a, w0, __uint_as_float((uint32_t)(k0 >> 32)), inv, nx, ny, nz, scale, acc);
            if (has1) est_add32w(a, w1, __uint_as_float((uint32_t)(k1 >> 32)), inv, nx, ny, nz, scale, acc);
        }
        acc.c0 = gsum_i64<G>(acc.c0, gmask);
        acc.c1 = gsum_i64<G>(acc.c1, gmask);
        acc.c2 = gsum_i64<G>(acc.c2, gmask);
        acc.f0 = __reduce_add_sync(gmask, acc.f0);
        acc.f1 = __reduce_add_sync(gmask, acc.f1);
        acc.f2 = __reduce_add_sync(gmask, acc.f2);
        double r2d = (double)r2;
        if (est_needs_fp64(a.filter, acc)) {
            if (kFix) {
                r2d = est_fp64_group<G>(a, buf, n, s, gmask, qx, qy, qz, nx, ny, nz, acc);
            } else if (s == 0) {   // re-evaluated by the fix pass (the FP32 result written below is replaced)
                a.fix_list[atomicAdd(a.fix_count, 1u)] = slot;
            }
        }
        rad = est_result(acc, r2d, scale, n, a.norm_c);
    }
    if (s == 0) {
        a.out_rad[qo] = rad;
        if (a.out_r2) a.out_r2[qo] = r2;
        if (a.out_count) a.out_count[qo] = n;
    }
    if (a.out_nbr)
        write_neighbours<G>(buf, n, s, gmask, a.pos, a.out_nbr + a.nbr_off + (size_t)(qo - a.q_off) * k, k, a.ph_off);
    return r2;
}

// ------------------------------------------------------------------------
// 32-wide tree traversal for one query held by a whole warp (G = 32): lane i
// tests child i of a wide node, passing internal children are pushed with the
// nearest on top, passing leaves are scanned in tree order (one photon per
// lane).  Candidates go to buf as in the binary traversal.
constexpr int kWideStack = 192;   // entries of 2 words: first child slot, stack_word(lower bound, child count)
// Single-map wide instances stage the root wide node's child slots (the top
// kWideLevels binary levels of the tree) in shared memory, once per block:
// every query visits them first.
constexpr int kTopBytes = 32 * (int)sizeof(ChildSlot);

// The search's threshold test is strict until a selection has run and
// inclusive after (x < thr, then x <= thr).  For the non-negative bounds and
// distances compared, x <= thr is x < the next float above thr, so one
// exclusive bound gives both as a single comparison.
__device__ __forceinline__ float excl_bound(float thr, bool selected) {
    return (selected && thr < INFINITY) ? __uint_as_float(__float_as_uint(thr) + 1u) : thr;
}

// One 32-photon half of a leaf: this lane's photon at tree position idx,
// at squared distance d2 from the query, when `have`.
__device__ __forceinline__ void scan_half(const KnnArgs& a, float d2, bool have, uint32_t idx, uint32_t k, uint32_t C,
                                          uint64_t* buf, uint32_t& n, bool& selected, float& thr, uint32_t* hist,
                                          uint32_t lane, uint32_t lt) {
    if (n + 32 > C) {   // make room: keep the k nearest, tighten the threshold
        const uint64_t T = group_select<32>(buf, n, k, hist, a.pos, lane, kFull, lt, thr);
        selected = true;
        thr = __uint_as_float((uint32_t)(T >> 32));
    }
    const bool acc = have && d2 < excl_bound(thr, selected);
    const uint32_t bal = __ballot_sync(kFull, acc);
    // appends only; readers of the buffer (a selection, the finish) sync before they read
    if (acc) buf[n + __popc(bal & lt)] = ((uint64_t)__float_as_uint(d2) << 32) | idx;
    n += __popc(bal);
}

// A leaf of up to 64 photons: both halves' loads are issued before either is
// tested, so a large leaf costs one load latency, and both distances are
// formed at once (the second half then holds one register, not a photon).
// Leaves of 64 (the autotuned size of the plain workload) against 32:
// 12.5 -> about 7.7 leaves per query for 23 % more photons tested, kernel
// 6.90 -> 6.52 ms.
__device__ __forceinline__ void scan_leaf(const KnnArgs& a, uint32_t ref, uint32_t cnt, float qx, float qy, float qz,
                                          uint32_t k, uint32_t C, uint64_t* buf, uint32_t& n, bool& selected,
                                          float& thr, uint32_t* hist, uint32_t lane, uint32_t lt) {
    float4 m0 = make_float4(0.f, 0.f, 0.f, 0.f), m1 = m0;
    if (lane < cnt) m0 = __ldg(a.pos + ref + lane);
    if (lane + 32 < cnt) m1 = __ldg(a.pos + ref + 32 + lane);
    const float d0 = d2_rn(qx, qy, qz, m0.x, m0.y, m0.z);
    const float d1 = d2_rn(qx, qy, qz, m1.x, m1.y, m1.z);
    scan_half(a, d0, lane < cnt, ref + lane, k, C, buf, n, selected, thr, hist, lane, lt);
    if (cnt > 32) scan_half(a, d1, lane + 32 < cnt, ref + 32 + lane, k, C, buf, n, selected, thr, hist, lane, lt);
}

// Stack entry of the wide traversal: two words, the wide node's first child
// slot and its lower bound with the 6 low mantissa bits replaced by the child
// count (<= 32).  Clearing those bits rounds the non-negative bound toward
// zero, so it stays a lower bound: a pop may visit a node the exact bound
// would skip, never the reverse.
__device__ __forceinline__ uint32_t stack_word(float lb, uint32_t kids) { return (__float_as_uint(lb) & ~63u) | kids; }

__device__ __forceinline__ void wide_traverse(const KnnArgs& a, float qx, float qy, float qz, uint32_t k, uint32_t C, uint64_t* buf,
                              uint32_t& n, bool& selected, float& thr, uint32_t* hist, uint32_t* stack, uint32_t lane,
                              uint32_t lt) {
    int sp = 0;
    {
        float lo[3], hi[3];
        uint32_t ref, cnt;
        load_root(a.root, lo, hi, ref, cnt);
        if (ref == kInvalid) return;
        const float lb = box_lb(qx, qy, qz, lo, hi);
        if (!(lb < excl_bound(thr, selected))) return;
        if (cnt & kWideFlag) {
            if (lane == 0) reinterpret_cast<uint2*>(stack)[0] = make_uint2(ref, stack_word(lb, cnt & kWideCount));
            sp = 1;
            __syncwarp();
        } else if (cnt > 0) {
            scan_leaf(a, ref, cnt, qx, qy, qz, k, C, buf, n, selected, thr, hist, lane, lt);
            return;
        }
    }
    while (sp > 0) {
        --sp;
        const uint2 entry = reinterpret_cast<const uint2*>(stack)[sp];
        const uint32_t first = entry.x, e1 = entry.y;
        const uint32_t kids = e1 & 63u;
        const float plb = __uint_as_float(e1 & ~63u);
        __syncwarp();
        const float thx = excl_bound(thr, selected);   // the node's children are tested against the same bound
        if (!(plb < thx)) continue;
        float lo[3], hi[3];
        uint32_t ref = kInvalid, cnt = 0;
        if (lane < kids) {
            if (first == a.top_first) {   // the root wide node: staged in shared memory
                const float4* tp = reinterpret_cast<const float4*>(a.s_top + lane);
                const float4 ta = tp[0], tb = tp[1];
                lo[0] = ta.x; lo[1] = ta.y; lo[2] = ta.z; hi[0] = ta.w;
                hi[1] = tb.x; hi[2] = tb.y; ref = __float_as_uint(tb.z); cnt = __float_as_uint(tb.w);
            } else {
                load_root(a.wchild + first + lane, lo, hi, ref, cnt);
            }
        }
        float lb = INFINITY;
        bool pass = false;
        if (ref != kInvalid) {
            lb = box_lb(qx, qy, qz, lo, hi);
            pass = lb < thx;
        }
        const bool is_wide = (cnt & kWideFlag) != 0;
        const uint32_t intm = __ballot_sync(kFull, pass && is_wide);
        const uint32_t leafm = __ballot_sync(kFull, pass && !is_wide);
        if (intm) {
            const uint32_t np = __popc(intm);
            if (sp + (int)np > kWideStack) {
                if (lane == 0) atomicOr(&a.hdr->errors, kErrStack);
            } else {
                // The nearest passing child (smallest lower bound, ties to the
                // lowest lane) goes on top: the bounds are non-negative, so their
                // bits order as the values, and one warp min-reduction finds it.
                const uint32_t lbb = ((intm >> lane) & 1u) ? __float_as_uint(lb) : 0xffffffffu;
                const uint32_t mn = __reduce_min_sync(kFull, lbb);
                const uint32_t near = (uint32_t)(__ffs(__ballot_sync(kFull, lbb == mn)) - 1);
                const uint32_t others = intm & ~(1u << near);
                if ((intm >> lane) & 1u) {
                    const uint32_t at = (uint32_t)sp + (lane == near ? np - 1 : __popc(others & lt));
                    reinterpret_cast<uint2*>(stack)[at] = make_uint2(ref, stack_word(lb, cnt & kWideCount));
                }
                sp += (int)np;
                __syncwarp();
            }
        }
        // Passing leaves in tree order: the threshold only changes when a
        // selection makes room (about once in five queries before the final
        // one), so ordering them by distance costs more than it saves
        // (measured 8.83 -> 8.35 ms); internal children keep the nearest on
        // top, which does pay.
        uint32_t rest = leafm;
        if (rest) {
            uint32_t b = __ffs(rest) - 1;
            const float thr0 = thr;
            for (;;) {
                const uint32_t lref = __shfl_sync(kFull, ref, b), lcnt = __shfl_sync(kFull, cnt, b);
                bool go = true;
                if (thr != thr0) {   // a selection tightened the threshold since the ballot
                    const float llb = __shfl_sync(kFull, lb, b);
                    go = llb <= thr;
                }
                if (go)
                    scan_leaf(a, lref, lcnt, qx, qy, qz, k, C, buf, n, selected, thr, hist, lane, lt);
                rest &= ~(1u << b);
                if (!rest) break;
                b = __ffs(rest) - 1;
            }
        }
    }
}

// The wide instances are held to 64 registers (4 blocks of 256 per SM, 32
// warps): measured fastest.  Without a bound ptxas holds them to 48
// registers and spills; with 3 blocks (80 registers, no spills, 24 warps) the
// plain workload's kernel took 8.19 ms against 6.95.
template <int G, bool kFix, bool kBatch, bool kWide>
__global__ void __launch_bounds__(256, kWide ? 4 : 0) k_knn_group(KnnArgs a0) {
    constexpr int QW = 32 / G;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = lane_id();
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t g = lane / G, s = lane % G;
    const uint32_t gbase = g * G;
    const uint32_t gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << gbase);
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t C = a0.cap;
    constexpr size_t top_off = (kWide && !kBatch) ? kTopBytes : 0;
    if constexpr (kWide && !kBatch) {   // stage the root wide node's children
        ChildSlot* st = reinterpret_cast<ChildSlot*>(smem);
        const ChildSlot r = *a0.root;
        const bool w = r.ref != kInvalid && (r.cnt & kWideFlag);
        if (w && threadIdx.x < (r.cnt & kWideCount)) st[threadIdx.x] = a0.wchild[r.ref + threadIdx.x];
        __syncthreads();
        a0.s_top = st;
        a0.top_first = w ? r.ref : kInvalid;
    }
    unsigned char* wb = smem + top_off + (size_t)warp * a0.smem_per_warp;
    uint64_t* buf = reinterpret_cast<uint64_t*>(wb) + (size_t)g * C;
    uint32_t* hist = reinterpret_cast<uint32_t*>(wb + (size_t)QW * C * sizeof(uint64_t)) + g * 256;
    uint32_t* stack = reinterpret_cast<uint32_t*>(wb + (size_t)QW * (C * sizeof(uint64_t) + 256 * sizeof(uint32_t)));
    const uint32_t nq = kFix ? *a0.nq_dev : a0.nq;
    const uint32_t total_rounds = (nq + QW - 1) / QW;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);

    for (;;) {
        uint32_t chunk = 0;
        if (lane == 0) chunk = atomicAdd(a0.work_counter, 1u);
        chunk = __shfl_sync(kFull, chunk, 0);
        uint32_t rbegin = 0, rlen = 0;
        if (!guided_chunk(chunk, total_rounds, nwarps, a0.rounds_per_chunk,
                          kBatch ? 4u * a0.rounds_per_chunk : 0xffffffffu, rbegin, rlen))
            break;
        float pqx = 0.f, pqy = 0.f, pqz = 0.f, pr = 0.f;
        bool pvalid = false;
        uint32_t pmap = 0;   // batch: map of the previous round's query
        for (uint32_t round = 0; round < rlen; ++round) {
            const uint32_t slot_q = (rbegin + round) * QW + g;
            const bool inrange = slot_q < nq;
            if (!__any_sync(kFull, inrange)) break;
            // per-query arguments: the launch's, or (batch) those of the query's map
            KnnArgs a = a0;
            uint32_t map = 0;
            const uint32_t slot_main = (kFix && inrange) ? a0.fix_in[slot_q] : slot_q;   // slot of the sorted launch
            if (kBatch && inrange) {
                map = (uint32_t)(a0.qkeys[slot_main] >> kBatchQueryMapShift);
                const BatchQuery bq = a0.bq[map];
                a.k = bq.k; a.r2max = bq.r2max; a.rmax = bq.rmax; a.filter = bq.filter; a.cone_k = bq.cone_k;
                a.min_found = bq.min_found; a.nbr_off = bq.nbr_off; a.q_off = bq.q_off; a.ph_off = bq.ph_off;
                a.norm_c = bq.norm_c;
                a.scale_ptr = &a0.bgeom[map].fix_scale;
                a.root = kWide ? &a0.bgeom[map].wroot : &a0.bgeom[map].root;
            }
            const uint32_t k = a.k;
            const float r2max = a.r2max;
            if (kBatch) {   // a radius bound only carries over within one map
                if (map != pmap) pvalid = false;
                pmap = map;
            }
            uint32_t qo = 0;
            float qx = 0.f, qy = 0.f, qz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
            bool active = false;
            if (inrange) {
                float4 q, nn;
                if (!kFix && !kBatch && a.qsorted) {   // records already in processing order
                    q = a.qsorted[2 * (size_t)slot_main];
                    nn = a.qsorted[2 * (size_t)slot_main + 1];
                    qo = __float_as_uint(q.w);
                } else {
                    qo = a.order ? a.order[slot_main] : slot_main;
                    q = a.qpos[qo];
                    nn = a.qnrm[qo];
                }
                qx = q.x; qy = q.y; qz = q.z;
                nx = nn.x; ny = nn.y; nz = nn.z;
                active = isfinite(qx) && isfinite(qy) && isfinite(qz);
                if (!active && s == 0) atomicOr(&a.hdr->errors, kErrQueryNonFinite);
            }
            // radius bound from the previous round's queries of this warp
            float tau0 = r2max;
#pragma unroll
            for (int h = 0; h < QW; ++h) {
                // one query per warp: every lane already holds its predecessor's values
                const int src = h * G;
                const float sx = QW == 1 ? pqx : __shfl_sync(kFull, pqx, src);
                const float sy = QW == 1 ? pqy : __shfl_sync(kFull, pqy, src);
                const float sz = QW == 1 ? pqz : __shfl_sync(kFull, pqz, src);
                const float sr = QW == 1 ? pr : __shfl_sync(kFull, pr, src);
                const bool sv = QW == 1 ? pvalid : __shfl_sync(kFull, pvalid, src);
                if (sv) {
                    const float dq = __fsqrt_rn(d2_rn(qx, qy, qz, sx, sy, sz));
                    const float b = __fmul_rn(__fadd_rn(sr, dq), 1.000244140625f);
                    tau0 = fminf(tau0, __fmul_rn(__fmul_rn(b, b), 1.000244140625f));
                }
            }
            uint32_t n = 0;          // entries in this group's buffer
            bool selected = false;   // a selection has run: threshold is inclusive
            float thr = tau0;
            bool todo = active;
            uint32_t st_nodes = 0, st_leaves = 0, st_photons = 0, st_cand = 0, st_sel = 0, st_redo = 0;
            while (__any_sync(kFull, todo)) {
                const bool live = todo;
                if (live) { n = 0; selected = false; thr = tau0; }
                if constexpr (kWide) {
                    if (live) wide_traverse(a, qx, qy, qz, k, C, buf, n, selected, thr, hist, stack, lane, lt);
                } else {
                int sp = 0;
                float lo[3], hi[3];
                uint32_t ref, cnt;
                load_root(a.root, lo, hi, ref, cnt);
                bool have;
                {
                    const float lb = box_lb(qx, qy, qz, lo, hi);
                    have = __any_sync(kFull, live && lb < thr) && ref != kInvalid;
                }
                for (;;) {
                    if (have) {
                        if (cnt > 0) {
                            ++st_leaves;
                            st_photons += cnt;
                            for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {   // 32 photons of the leaf at a time
                                float4 mine = make_float4(0.f, 0.f, 0.f, 0.f);
                                if (c0 + lane < cnt) mine = __ldg(a.pos + ref + c0 + lane);
                                const uint32_t cn = min(cnt - c0, 32u);
                                for (uint32_t j0 = 0; j0 < cn; j0 += G) {
                                    // make room: a group whose buffer cannot take G more entries selects first
                                    const bool full = live && (n + G > C);
                                    if (__any_sync(kFull, full)) {
                                        if (full) {
                                            const uint64_t T = group_select<G>(buf, n, k, hist, a.pos, s, gmask, lt, thr);
                                            ++st_sel;
                                            selected = true;
                                            thr = __uint_as_float((uint32_t)(T >> 32));
                                        }
                                        __syncwarp();
                                    }
                                    const uint32_t j = j0 + s;
                                    const uint32_t src = j < 32 ? j : 31;
                                    const float px = __shfl_sync(kFull, mine.x, src);
                                    const float py = __shfl_sync(kFull, mine.y, src);
                                    const float pz = __shfl_sync(kFull, mine.z, src);
                                    bool acc = false;
                                    float d2 = 0.f;
                                    if (live && j < cn) {
                                        d2 = d2_rn(qx, qy, qz, px, py, pz);
                                        acc = selected ? (d2 <= thr) : (d2 < thr);
                                    }
                                    const uint32_t bal = __ballot_sync(kFull, acc) & gmask;
                                    if (acc) buf[n + __popc(bal & lt)] = ((uint64_t)__float_as_uint(d2) << 32) | (ref + c0 + j);
                                    n += __popc(bal);
                                    st_cand += __popc(bal);
                                }
                            }
                            __syncwarp();
                            have = false;
                        } else {
                            ++st_nodes;
                            float l0[3], h0[3], l1[3], h1[3];
                            uint32_t r0, c0, r1, c1;
                            load_slot(a.nodes, ref, 0, l0, h0, r0, c0);
                            load_slot(a.nodes, ref, 1, l1, h1, r1, c1);
                            const float lb0 = box_lb(qx, qy, qz, l0, h0);
                            const float lb1 = box_lb(qx, qy, qz, l1, h1);
                            const bool p0 = live && (selected ? lb0 <= thr : lb0 < thr);
                            const bool p1 = live && (selected ? lb1 <= thr : lb1 < thr);
                            const uint32_t b0 = __ballot_sync(kFull, p0), b1 = __ballot_sync(kFull, p1);
                            const bool w0 = b0 != 0 && r0 != kInvalid, w1 = b1 != 0 && r1 != kInvalid;
                            if (w0 && w1) {
                                const uint32_t votes = __ballot_sync(kFull, (p0 || p1) && lb1 < lb0);
                                const int near = (2 * __popc(votes) > __popc(b0 | b1)) ? 1 : 0;
                                if (sp >= kStackDepth) {
                                    if (lane == 0) atomicOr(&a.hdr->errors, kErrStack);
                                } else {
                                    if (lane == 0) stack[sp] = (ref << 1) | (uint32_t)(1 - near);
                                    ++sp;
                                }
                                if (near) { ref = r1; cnt = c1; } else { ref = r0; cnt = c0; }
                            } else if (w0) {
                                ref = r0; cnt = c0;
                            } else if (w1) {
                                ref = r1; cnt = c1;
                            } else {
                                have = false;
                            }
                        }
                        continue;
                    }
                    bool found = false;
                    while (sp > 0) {
                        --sp;
                        __syncwarp();
                        const uint32_t e = stack[sp];
                        load_slot(a.nodes, e >> 1, e & 1u, lo, hi, ref, cnt);
                        const float lb = box_lb(qx, qy, qz, lo, hi);
                        const bool p = live && (selected ? lb <= thr : lb < thr);
                        if (__any_sync(kFull, p)) { found = true; break; }
                    }
                    if (!found) break;
                    have = true;
                }
                }
                // the bound admitted fewer than k photons: redo this query with R
                todo = live && n < k && tau0 < r2max;
                if (todo) { tau0 = r2max; ++st_redo; }
                __syncwarp();
            }
            // final selection and epilogue (group-local from here on)
            float rk2 = r2max;
            if (!kWide && a.stats && s == 0 && active) {   // binary layouts only: no counters in the wide instances
                atomicAdd(a.stats + kStatQueries, 1ull);
                atomicAdd(a.stats + kStatCandidates, (unsigned long long)st_cand);
                atomicAdd(a.stats + kStatSelections, (unsigned long long)(st_sel + (n > k ? 1 : 0)));
                atomicAdd(a.stats + kStatRedo, (unsigned long long)st_redo);
                if (!pvalid_any_bound(tau0, r2max, st_redo)) atomicAdd(a.stats + kStatUnbounded, 1ull);
            }
            if (!kWide && a.stats && lane == 0) {
                atomicAdd(a.stats + kStatNodes, (unsigned long long)st_nodes);
                atomicAdd(a.stats + kStatLeaves, (unsigned long long)st_leaves);
                atomicAdd(a.stats + kStatPhotons, (unsigned long long)st_photons);
            }
            if (active) {
                const float r2 = group_finish<G, kFix>(a, buf, n, hist, thr, s, gmask, lt, qo, slot_main, qx, qy, qz, nx, ny, nz);
                rk2 = r2;
            } else if (inrange && s == 0) {
                a.out_rad[qo] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (a.out_r2) a.out_r2[qo] = r2max;
                if (a.out_count) a.out_count[qo] = 0;
            }
            if (inrange && !active && a.out_nbr)
                for (uint32_t j = s; j < k; j += G) a.out_nbr[a.nbr_off + (size_t)(qo - a.q_off) * k + j] = kInvalid;
            __syncwarp();
            pqx = qx; pqy = qy; pqz = qz;
            pvalid = active && n == k;
            pr = pvalid ? __fsqrt_rn(rk2) : 0.0f;
        }
    }
}

// Brute force: thread per query, every photon staged through shared memory.
constexpr int kBruteThreads = 64;
constexpr int kBruteTile = 512;

__global__ void __launch_bounds__(kBruteThreads) k_knn_brute(KnnArgs a, uint32_t n) {
    extern __shared__ __align__(16) unsigned char smem[];
    float4* tile = reinterpret_cast<float4*>(smem);
    uint64_t* heap = reinterpret_cast<uint64_t*>(smem + kBruteTile * sizeof(float4)) + threadIdx.x;
    const uint32_t q = blockIdx.x * kBruteThreads + threadIdx.x;
    const bool valid = q < a.nq;
    float qx = 0.f, qy = 0.f, qz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
    if (valid) {
        const float4 p = a.qpos[q], nn = a.qnrm[q];
        qx = p.x; qy = p.y; qz = p.z; nx = nn.x; ny = nn.y; nz = nn.z;
    }
    uint32_t hn = 0;
    uint64_t top = 0;
    const uint32_t k = a.k;
    // the heap helpers use a stride of 32; this kernel uses its own stride
    for (uint32_t base = 0; base < n; base += kBruteTile) {
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < kBruteTile && base + t < n; t += kBruteThreads) tile[t] = a.pos[base + t];
        __syncthreads();
        const uint32_t lim = min((uint32_t)kBruteTile, n - base);
        if (!valid) continue;
        for (uint32_t t = 0; t < lim; ++t) {
            const float4 p = tile[t];
            const float d2 = d2_rn(qx, qy, qz, p.x, p.y, p.z);
            if (!(d2 < a.r2max)) continue;
            const uint64_t key = ((uint64_t)__float_as_uint(d2) << 32) | (base + t);
            if (hn < k) {
                uint32_t i = hn++;
                while (i > 0) {
                    const uint32_t pi = (i - 1) >> 1;
                    const uint64_t pv = heap[pi * kBruteThreads];
                    if (!key_less(pv, key, a.pos)) break;
                    heap[i * kBruteThreads] = pv;
                    i = pi;
                }
                heap[i * kBruteThreads] = key;
                top = heap[0];
            } else if (key_less(key, top, a.pos)) {
                uint32_t i = 0;
                for (;;) {
                    const uint32_t l = 2 * i + 1;
                    if (l >= k) break;
                    uint32_t c = l;
                    uint64_t cv = heap[l * kBruteThreads];
                    if (l + 1 < k) {
                        const uint64_t rv = heap[(l + 1) * kBruteThreads];
                        if (key_less(cv, rv, a.pos)) { c = l + 1; cv = rv; }
                    }
                    if (!key_less(key, cv, a.pos)) break;
                    heap[i * kBruteThreads] = cv;
                    i = c;
                }
                heap[i * kBruteThreads] = key;
                top = heap[0];
            }
        }
    }
    if (valid) finish_query(a, heap, kBruteThreads, hn, q, qx, qy, qz, nx, ny, nz);
}

// Query records in processing order: rec[2i] = (position xyz, caller index
// bits), rec[2i + 1] = normal of query order[i].
__global__ void k_gather_queries(const uint32_t* __restrict__ order, const float4* __restrict__ qpos,
                                 const float4* __restrict__ qnrm, uint32_t nq, float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const uint32_t o = order[i];
    float4 p = qpos[o];
    p.w = __uint_as_float(o);
    out[2 * (size_t)i] = p;
    out[2 * (size_t)i + 1] = qnrm[o];
}

int gather_queries(const uint32_t* order, const float4* qpos, const float4* qnrm, uint32_t nq, float4* out,
                   cudaStream_t st) {
    if (!nq) return 0;
    k_gather_queries<<<(nq + 255) / 256, 256, 0, st>>>(order, qpos, qnrm, nq, out);
    return 1;
}

// Processing-order keys of the queries: a 30-bit Hilbert index (the kNN
// query, a warp per query, profits from consecutive queries being neighbours)
// or a 30-bit Morton code (the cut interpolation, a thread per query, profits
// from a warp's 32 queries filling compact Morton blocks: 0.654 -> 0.587 ms
// against Hilbert order on the plain workload).
template <bool kHilbert>
__global__ void k_query_order(const float4* __restrict__ qpos, uint32_t nq, const MapHeader* __restrict__ hdr,
                              uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const float ext = fmaxf(fmaxf(__fsub_rn(hdr->hi[0], hdr->lo[0]), __fsub_rn(hdr->hi[1], hdr->lo[1])),
                            __fsub_rn(hdr->hi[2], hdr->lo[2]));
    const float scale = (ext > 0.0f && isfinite(ext)) ? __fdiv_rn(65536.0f, ext) : 0.0f;
    const float4 p = qpos[i];
    keys[i] = kHilbert ? hilbert30(p.x, p.y, p.z, hdr->lo, scale) : morton30(p.x, p.y, p.z, hdr->lo, scale);
    vals[i] = i;
}

// 30-bit query keys (Hilbert, or Morton when hilbert is false): 4 radix
// passes instead of the tree's 6 (a cell is 1/1024 of the map's extent per
// axis, finer than the query spacing of the measured workloads).
int query_order_keys(const float4* qpos, uint32_t nq, const MapHeader* hdr, uint32_t* keys, uint32_t* vals,
                     cudaStream_t st, bool hilbert) {
    if (!nq) return 0;
    if (hilbert) k_query_order<true><<<(nq + 255) / 256, 256, 0, st>>>(qpos, nq, hdr, keys, vals);
    else k_query_order<false><<<(nq + 255) / 256, 256, 0, st>>>(qpos, nq, hdr, keys, vals);
    return 1;
}

int query_smem_bytes_per_warp(uint32_t k) {
    return (int)(32 * k * sizeof(uint64_t) + kStackDepth * sizeof(uint32_t));
}

// The filter's normalisation constant c, the estimate's factor being c / r^2:
// 1 / ((1 - 2 / (3 k_c)) pi) (cone), 2 / pi (Epanechnikov), 1 / pi (box).
double filter_norm_const(int filter, float cone_k) {
    const double pi = 3.14159265358979323846;
    if (filter == 1) return 1.0 / ((1.0 - 2.0 / (3.0 * (double)cone_k)) * pi);
    if (filter == 2) return 2.0 / pi;
    return 1.0 / pi;
}

static KnnArgs make_args(const MapView& m, const QueryParams& p, const float4* qpos, const float4* qnrm,
                         const uint32_t* order, uint32_t nq, const QueryOutputs& out) {
    KnnArgs a;
    a.pos = m.pos; a.pow = m.pow; a.nodes = m.nodes; a.hdr = m.hdr;
    a.qpos = qpos; a.qnrm = qnrm; a.order = order; a.nq = nq;
    a.k = p.k; a.r2max = p.r2; a.rmax = p.r; a.filter = p.filter; a.cone_k = p.cone_k; a.min_found = p.min_found;
    a.out_rad = out.rad; a.out_nbr = out.nbr; a.out_r2 = out.r2; a.out_count = out.count;
    a.work_counter = nullptr; a.rounds_per_chunk = 1;
    a.fix_list = nullptr; a.fix_count = nullptr; a.nq_dev = nullptr; a.fix_in = nullptr;
    a.scale_ptr = &m.hdr->fix_scale;
    a.root = &m.nodes[0].c[0];
    a.wchild = m.wchild;
    a.nbr_off = 0; a.q_off = 0; a.ph_off = 0;
    a.qkeys = nullptr; a.bgeom = nullptr; a.bq = nullptr;
    a.cap = 0; a.smem_per_warp = 0; a.stats = nullptr;
    a.norm_c = filter_norm_const(p.filter, p.cone_k);
    a.qsorted = nullptr;
    a.s_top = nullptr; a.top_first = kInvalid;
    return a;
}

// Candidate buffer entries per query: k rounded up to a warp, plus 96 of
// headroom before a selection must make room (with leaves of up to 64
// photons, 96 measured 5.90 -> 5.87 ms against 64 on the plain workload).
uint32_t group_capacity(uint32_t k) { return ((k + 31u) & ~31u) + 96u; }

int wide_smem_bytes_per_warp(uint32_t k) {
    return (int)(group_capacity(k) * sizeof(uint64_t) + 256 * sizeof(uint32_t)) + 2 * kWideStack * (int)sizeof(uint32_t);
}

int group_smem_bytes_per_warp(uint32_t k, int qpw) {
    return qpw * (int)(group_capacity(k) * sizeof(uint64_t) + 256 * sizeof(uint32_t)) +
           kStackDepth * (int)sizeof(uint32_t);
}

template <class K>
static uint32_t grid_for(K kernel, int threads, int smem, uint32_t work_items, int warps_per_block) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (per_sm < 1) per_sm = 1;
    uint32_t grid = (uint32_t)(sms * per_sm);
    const uint32_t need = (work_items + warps_per_block - 1) / warps_per_block;
    return grid > need ? need : (grid ? grid : 1);
}

int query_knn(const MapView& m, const QueryParams& p, const float4* qpos, const float4* qnrm,
              const uint32_t* order, uint32_t nq, const QueryOutputs& out, uint32_t* work_counter, uint32_t* fix_list,
              const QueryTuning& t, cudaStream_t st) {
    if (!nq) return 0;
    KnnArgs a = make_args(m, p, qpos, qnrm, order, nq, out);
    a.work_counter = work_counter;
    a.stats = t.stats;
    if (t.stats) cudaMemsetAsync(t.stats, 0, kStatCount * sizeof(unsigned long long), st);
    a.rounds_per_chunk = (uint32_t)t.rounds_per_chunk;
    const int threads = 32 * t.warps_per_block;
    cudaMemsetAsync(work_counter, 0, 3 * sizeof(uint32_t), st);   // work, fix count, fix work
    if (t.layout == 0) {   // one lane per query, shared-memory heap
        const int smem = query_smem_bytes_per_warp(p.k) * t.warps_per_block;
        const uint32_t nchunks = (nq + 32u * a.rounds_per_chunk - 1) / (32u * a.rounds_per_chunk);
        const uint32_t grid = grid_for(k_knn_tree, threads, smem, nchunks, t.warps_per_block);
        k_knn_tree<<<grid, threads, smem, st>>>(a);
        return 1;
    }
    if (t.layout == 2) {   // one query per warp over the 32-wide tree
        a.qsorted = t.qsorted;
        a.cap = group_capacity(p.k);
        a.smem_per_warp = (uint32_t)wide_smem_bytes_per_warp(p.k);
        a.root = m.wroot;
        a.fix_list = fix_list;
        a.fix_count = work_counter + 1;
        const int smem = (int)a.smem_per_warp * t.warps_per_block + kTopBytes;
        const uint32_t nchunks = (nq + a.rounds_per_chunk - 1) / a.rounds_per_chunk;
        KnnArgs fx = a;
        fx.fix_in = fix_list;
        fx.nq_dev = work_counter + 1;
        fx.work_counter = work_counter + 2;
        fx.qsorted = nullptr;
        const uint32_t grid = grid_for(k_knn_group<32, false, false, true>, threads, smem, nchunks, t.warps_per_block);
        k_knn_group<32, false, false, true><<<grid, threads, smem, st>>>(a);
        const uint32_t gfix = grid_for(k_knn_group<32, true, false, true>, threads, smem, nchunks, t.warps_per_block);
        k_knn_group<32, true, false, true><<<gfix, threads, smem, st>>>(fx);
        return 2;
    }
    const int qpw = t.queries_per_warp;
    a.cap = group_capacity(p.k);
    a.smem_per_warp = (uint32_t)group_smem_bytes_per_warp(p.k, qpw);
    const int smem = (int)a.smem_per_warp * t.warps_per_block;
    const uint32_t nchunks = (nq + (uint32_t)qpw * a.rounds_per_chunk - 1) / ((uint32_t)qpw * a.rounds_per_chunk);
    a.fix_list = fix_list;
    a.fix_count = work_counter + 1;
    a.nq_dev = nullptr;
    KnnArgs fx = a;   // fix pass: the listed queries, FP64 distances where needed
    fx.fix_in = fix_list;
    fx.nq_dev = work_counter + 1;
    fx.work_counter = work_counter + 2;
#define PM_LAUNCH_GROUP(G)                                                                          \
    {                                                                                               \
        const uint32_t grid = grid_for(k_knn_group<G, false, false, false>, threads, smem, nchunks, t.warps_per_block); \
        k_knn_group<G, false, false, false><<<grid, threads, smem, st>>>(a);                                      \
        const uint32_t gfix = grid_for(k_knn_group<G, true, false, false>, threads, smem, nchunks, t.warps_per_block); \
        k_knn_group<G, true, false, false><<<gfix, threads, smem, st>>>(fx);                                      \
    }
    switch (qpw) {
        case 1: PM_LAUNCH_GROUP(32) break;
        case 2: PM_LAUNCH_GROUP(16) break;
        case 4: PM_LAUNCH_GROUP(8) break;
        default: PM_LAUNCH_GROUP(4) break;
    }
#undef PM_LAUNCH_GROUP
    return 2;
}

// One persistent launch over the queries of many maps (one query per warp):
// the sorted query keys carry each query's map id, whose root slot and
// parameters the kernel reads; kmax sizes the candidate buffers.
template <bool kW>
static int launch_batch(const MapView& m, const BatchQuery* bq, const BatchGeom* bg, uint32_t kmax, const float4* qpos,
                    const float4* qnrm, const uint32_t* order, const uint64_t* qkeys, uint32_t nq,
                    const QueryOutputs& out, uint32_t* work_counter, uint32_t* fix_list, const QueryTuning& t,
                    cudaStream_t st) {
    if (!nq) return 0;
    QueryParams p;
    p.k = kmax; p.r = 0.0f; p.r2 = 0.0f; p.filter = 0; p.cone_k = 1.0f; p.min_found = 0;
    KnnArgs a = make_args(m, p, qpos, qnrm, order, nq, out);
    a.work_counter = work_counter;
    a.rounds_per_chunk = (uint32_t)t.rounds_per_chunk;
    a.qkeys = qkeys;
    a.bgeom = bg;
    a.bq = bq;
    a.cap = group_capacity(kmax);
    a.smem_per_warp = (uint32_t)(kW ? wide_smem_bytes_per_warp(kmax) : group_smem_bytes_per_warp(kmax, 1));
    a.fix_list = fix_list;
    a.fix_count = work_counter + 1;
    const int threads = 32 * t.warps_per_block;
    const int smem = (int)a.smem_per_warp * t.warps_per_block;
    cudaMemsetAsync(work_counter, 0, 3 * sizeof(uint32_t), st);
    const uint32_t nchunks = (nq + a.rounds_per_chunk - 1) / a.rounds_per_chunk;
    const uint32_t grid = grid_for(k_knn_group<32, false, true, kW>, threads, smem, nchunks, t.warps_per_block);
    k_knn_group<32, false, true, kW><<<grid, threads, smem, st>>>(a);
    KnnArgs fx = a;   // queries whose estimate needs FP64 distances
    fx.fix_in = fix_list;
    fx.nq_dev = work_counter + 1;
    fx.work_counter = work_counter + 2;
    const uint32_t gfix = grid_for(k_knn_group<32, true, true, kW>, threads, smem, nchunks, t.warps_per_block);
    k_knn_group<32, true, true, kW><<<gfix, threads, smem, st>>>(fx);
    return 2;
}

int query_knn_batch(const MapView& m, const BatchQuery* bq, const BatchGeom* bg, uint32_t kmax, const float4* qpos,
                    const float4* qnrm, const uint32_t* order, const uint64_t* qkeys, uint32_t nq,
                    const QueryOutputs& out, uint32_t* work_counter, uint32_t* fix_list, const QueryTuning& t,
                    cudaStream_t st) {
    if (t.layout == 2)
        return launch_batch<true>(m, bq, bg, kmax, qpos, qnrm, order, qkeys, nq, out, work_counter, fix_list, t, st);
    return launch_batch<false>(m, bq, bg, kmax, qpos, qnrm, order, qkeys, nq, out, work_counter, fix_list, t, st);
}

int query_bruteforce(const MapView& m, const QueryParams& p, const float4* qpos, const float4* qnrm,
                     uint32_t nq, const QueryOutputs& out, cudaStream_t st) {
    if (!nq) return 0;
    KnnArgs a = make_args(m, p, qpos, qnrm, nullptr, nq, out);
    const int smem = kBruteTile * (int)sizeof(float4) + kBruteThreads * (int)p.k * (int)sizeof(uint64_t);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_knn_brute, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_knn_brute<<<(nq + kBruteThreads - 1) / kBruteThreads, kBruteThreads, smem, st>>>(a, m.n);
    return 1;
}

}  // namespace pm
