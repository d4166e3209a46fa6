// pm_build.cu -- point kd-tree build over photons.
//
// Replaces KDTreeGPU::BuildTree (KDTreeGPU.cpp:175-209) with its large-node
// stage (empty-space cuts, longest-axis spatial median, KDTreeGPU.cpp:444-664,
// GPU/kdtree.cu:467-824), small-node stage (KDTreeGPU.cpp:945-1154) and
// preorder layout pass (GPU/kdtree.cu:1658-1770).  The new build has no host
// synchronisation and a fixed launch sequence (graph-capturable):
//
//   1. k_bounds       photon bounds + largest flux channel (one pass, last
//                     block finalises the header)
//   2. k_morton       39-bit Morton code per photon in the cubic root cell
//   3. radix sort     (code, caller index): caller index breaks ties, so the
//                     order -- and the whole tree -- is deterministic
//                     (the reference picks sides of split-plane ties at
//                     random, GPU/kdtree.cu:806-815)
//   4. k_gather       photons into tree order as SoA float4 records, and the
//                     inverse permutation (caller index -> tree position)
//   5. k_radix_tree   binary radix tree over the sorted codes (Karras 2012):
//                     each internal node splits at the highest Morton bit
//                     that differs inside its range, i.e. at the spatial
//                     median of its cell on the axis that bit encodes
//                     (x, y, z in turn = the longest axis of a cube cell)
//   6. scan           keep flags of nodes holding more than leaf_size photons
//                     -> compacted node indices (stream compaction)
//   7. k_emit         64-byte nodes: two child slots, each a leaf range or an
//                     internal node, leaf boxes computed from their photons
//   8. k_refit        bottom-up child boxes (atomic arrival counters; boxes
//                     are min/max so the result is order independent)
#include "pm_internal.h"

namespace pm {

constexpr int kBoundsThreads = 256;
constexpr int kBoundsBlocksMax = 1184;   // 8 per SM on 148 SMs
constexpr int kLeafBoxBlocks = 1184;     // 8 blocks of 8 warps per SM, grid-stride over the nodes

// The wide tree's child-count scan in WideBuffers::scratch: ticket, total,
// one uint64 look-back word per tile of 256 nodes.
size_t wide_scan_words(uint32_t n) { return 2 + 2 * (size_t)((n + 255) / 256); }

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// partials: 8 words per block + one arrival counter at partials[8 * gridDim.x].
__global__ void __launch_bounds__(kBoundsThreads) k_bounds(const float4* __restrict__ pos,
                                                            const float4* __restrict__ pw, uint32_t n,
                                                            float* __restrict__ partials, MapHeader* hdr) {
    float v[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, 0.0f};
    uint32_t bad = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        const float4 w = pw[i];
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) { bad = 1; continue; }
        v[0] = fminf(v[0], p.x); v[1] = fminf(v[1], p.y); v[2] = fminf(v[2], p.z);
        v[3] = fmaxf(v[3], p.x); v[4] = fmaxf(v[4], p.y); v[5] = fmaxf(v[5], p.z);
        v[6] = fmaxf(v[6], fmaxf(fmaxf(fabsf(w.x), fabsf(w.y)), fabsf(w.z)));
    }
    __shared__ float s_v[kBoundsThreads / 32][8];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < 3; ++a) { v[a] = warp_min(v[a]); v[a + 3] = warp_max(v[a + 3]); }
    v[6] = warp_max(v[6]);
    bad = __any_sync(0xffffffffu, bad) ? 1u : 0u;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 7; ++a) s_v[warp][a] = v[a];
        s_v[warp][7] = __uint_as_float(bad);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBoundsThreads / 32; ++w) {
            for (int a = 0; a < 3; ++a) { s_v[0][a] = fminf(s_v[0][a], s_v[w][a]); s_v[0][a + 3] = fmaxf(s_v[0][a + 3], s_v[w][a + 3]); }
            s_v[0][6] = fmaxf(s_v[0][6], s_v[w][6]);
            s_v[0][7] = __uint_as_float(__float_as_uint(s_v[0][7]) | __float_as_uint(s_v[w][7]));
        }
        for (int a = 0; a < 8; ++a) partials[8 * blockIdx.x + a] = s_v[0][a];
        __threadfence();
        unsigned int* counter = reinterpret_cast<unsigned int*>(partials + 8 * gridDim.x);
        s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    // last block: all threads reduce the block partials, strided
    __threadfence();
    float r[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, 0.0f};
    uint32_t rb = 0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const float* q = partials + 8 * b;
        for (int a = 0; a < 3; ++a) { r[a] = fminf(r[a], __ldcg(q + a)); r[a + 3] = fmaxf(r[a + 3], __ldcg(q + a + 3)); }
        r[6] = fmaxf(r[6], __ldcg(q + 6));
        rb |= __float_as_uint(__ldcg(q + 7));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) { r[a] = warp_min(r[a]); r[a + 3] = warp_max(r[a + 3]); }
    r[6] = warp_max(r[6]);
    rb = __any_sync(0xffffffffu, rb != 0) ? 1u : 0u;
    __syncthreads();   // s_v is reused
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 7; ++a) s_v[warp][a] = r[a];
        s_v[warp][7] = __uint_as_float(rb);
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < kBoundsThreads / 32; ++w) {
        for (int a = 0; a < 3; ++a) { s_v[0][a] = fminf(s_v[0][a], s_v[w][a]); s_v[0][a + 3] = fmaxf(s_v[0][a + 3], s_v[w][a + 3]); }
        s_v[0][6] = fmaxf(s_v[0][6], s_v[w][6]);
        s_v[0][7] = __uint_as_float(__float_as_uint(s_v[0][7]) | __float_as_uint(s_v[w][7]));
    }
    for (int a = 0; a < 3; ++a) { r[a] = s_v[0][a]; r[a + 3] = s_v[0][a + 3]; }
    r[6] = s_v[0][6];
    rb = __float_as_uint(s_v[0][7]);
    for (int a = 0; a < 3; ++a) { hdr->lo[a] = r[a]; hdr->hi[a] = r[a + 3]; }
    hdr->max_power = r[6];
    hdr->fix_scale = fix_scale_of(r[6]);
    hdr->n = n;
    if (rb) atomicOr(&hdr->errors, kErrNonFinite);
    *reinterpret_cast<unsigned int*>(partials + 8 * gridDim.x) = 0u;   // ready for the next build
}

__device__ __forceinline__ float morton_scale(const MapHeader* hdr) {
    const float ext = fmaxf(fmaxf(__fsub_rn(hdr->hi[0], hdr->lo[0]), __fsub_rn(hdr->hi[1], hdr->lo[1])),
                            __fsub_rn(hdr->hi[2], hdr->lo[2]));
    return (ext > 0.0f && isfinite(ext)) ? __fdiv_rn(65536.0f, ext) : 0.0f;
}

__global__ void k_morton(const float4* __restrict__ pos, uint32_t n, const MapHeader* __restrict__ hdr,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float scale = morton_scale(hdr);
    const float4 p = pos[i];
    keys[i] = morton39(p.x, p.y, p.z, hdr->lo, scale);
    vals[i] = i;
}

__global__ void k_gather(const float4* __restrict__ pos, const float4* __restrict__ pw,
                         const uint32_t* __restrict__ order, uint32_t n, int format, float4* __restrict__ out_pos,
                         float4* __restrict__ out_pow, uint32_t* __restrict__ inv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t src = order[i];
    const float4 p = pos[src];
    const float4 w = pw[src];
    const uint32_t dir = (format == 0) ? spherical_to_oct(p.w, w.w) : __float_as_uint(w.w);
    out_pos[i] = make_float4(p.x, p.y, p.z, __uint_as_float(src));
    out_pow[i] = make_float4(w.x, w.y, w.z, __uint_as_float(dir));
    inv[src] = i;
}

// Common-prefix length of sorted codes i and j, caller index breaking ties.
__device__ __forceinline__ int delta(const uint64_t* __restrict__ keys, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = keys[i], b = keys[j];
    if (a != b) return __clzll(a ^ b);
    return 64 + __clz((uint32_t)i ^ (uint32_t)j);
}

// Thread per radix-tree node i (Karras 2012): direction, range [first, last],
// split, and the keep flag (more than leaf_size photons).
__global__ void k_radix_tree(const uint64_t* __restrict__ keys, uint32_t n, uint32_t leaf_size,
                             uint32_t* __restrict__ kfirst, uint32_t* __restrict__ klast,
                             uint32_t* __restrict__ ksplit, uint32_t* __restrict__ kkeep) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nn = n;
    if (i >= nn - 1) return;
    const int d = (delta(keys, nn, i, i + 1) > delta(keys, nn, i, i - 1)) ? 1 : -1;
    const int dmin = delta(keys, nn, i, i - d);
    int64_t lmax = 2;
    while (delta(keys, nn, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, nn, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(keys, nn, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(keys, nn, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
    const int64_t first = d > 0 ? i : j, last = d > 0 ? j : i;
    kfirst[i] = (uint32_t)first;
    klast[i] = (uint32_t)last;
    ksplit[i] = (uint32_t)gamma;
    kkeep[i] = (last - first + 1 > (int64_t)leaf_size) ? 1u : 0u;
}

__device__ __forceinline__ void leaf_box(const float4* __restrict__ pos, uint32_t first, uint32_t cnt, ChildSlot& s) {
    float lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY, hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY;
    for (uint32_t k = 0; k < cnt; ++k) {
        const float4 p = pos[first + k];
        lo0 = fminf(lo0, p.x); lo1 = fminf(lo1, p.y); lo2 = fminf(lo2, p.z);
        hi0 = fmaxf(hi0, p.x); hi1 = fmaxf(hi1, p.y); hi2 = fmaxf(hi2, p.z);
    }
    s.lo[0] = lo0; s.lo[1] = lo1; s.lo[2] = lo2;
    s.hi[0] = hi0; s.hi[1] = hi1; s.hi[2] = hi2;
}

__device__ __forceinline__ ChildSlot empty_slot() {
    ChildSlot s;
    s.lo[0] = s.lo[1] = s.lo[2] = INFINITY;
    s.hi[0] = s.hi[1] = s.hi[2] = -INFINITY;
    s.ref = kInvalid;
    s.cnt = 0;
    return s;
}

// Thread per radix-tree node; kept nodes write their compacted node.
__global__ void k_emit(const float4* __restrict__ pos, uint32_t n, uint32_t leaf_size,
                       const uint32_t* __restrict__ kfirst, const uint32_t* __restrict__ klast,
                       const uint32_t* __restrict__ ksplit, const uint32_t* __restrict__ kkeep,
                       const uint32_t* __restrict__ krank, const uint32_t* __restrict__ total, Node* __restrict__ nodes,
                       uint32_t* __restrict__ parent, uint32_t* __restrict__ arrive, uint32_t* __restrict__ nleaf,
                       MapHeader* hdr) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        const uint32_t m = (n > 1) ? *total : 0u;
        hdr->num_nodes = m;
        Node sr;
        sr.c[1] = empty_slot();
        if (n == 0) {
            sr.c[0] = empty_slot();
        } else if (m == 0) {   // whole map is one leaf
            ChildSlot s;
            leaf_box(pos, 0, n, s);
            s.ref = 0;
            s.cnt = n;
            sr.c[0] = s;
        } else {               // root box is filled in by k_refit
            sr.c[0] = empty_slot();
            sr.c[0].ref = 1;
            sr.c[0].cnt = 0;
        }
        nodes[0] = sr;
    }
    if (n < 2 || i >= (uint64_t)n - 1 || !kkeep[i]) return;
    const uint32_t id = 1 + krank[i];
    const uint32_t first = kfirst[i], last = klast[i], gamma = ksplit[i];
    Node nd;
    uint32_t leaves = 0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const uint32_t cf = side ? gamma + 1 : first;
        const uint32_t cl = side ? last : gamma;
        const uint32_t size = cl - cf + 1;
        ChildSlot s;
        if (size <= leaf_size) {   // box filled in by k_leaf_boxes
            s = empty_slot();
            s.ref = cf;
            s.cnt = size;
            ++leaves;
        } else {
            const uint32_t c = side ? gamma + 1 : gamma;   // radix-tree index of the internal child
            const uint32_t cid = 1 + krank[c];
            s = empty_slot();
            s.ref = cid;
            s.cnt = 0;
            parent[cid] = (id << 1) | (uint32_t)side;
        }
        nd.c[side] = s;
    }
    nodes[id] = nd;
    arrive[id] = leaves;
    nleaf[id] = leaves;
}

// Leaf boxes: warp per compacted node (grid-stride over nodes 1..m), lane i
// takes photon i of a leaf, min / max by warp reductions on order-preserving
// keys of the coordinates.
__device__ __forceinline__ uint32_t ord_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_float(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void k_leaf_boxes(const float4* __restrict__ pos, Node* __restrict__ nodes, const MapHeader* __restrict__ hdr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t m = hdr->num_nodes;
    for (uint32_t j = 1u + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); j <= m; j += warps) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const uint32_t cnt = nodes[j].c[side].cnt;
            if (cnt == 0) continue;
            const uint32_t ref = nodes[j].c[side].ref;
            float4 p = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
            float4 q = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
            if (lane < cnt) { p = pos[ref + lane]; q = p; }
            if (lane + 32 < cnt) {   // leaves hold up to kLeafMax = 64 photons
                const float4 r = pos[ref + 32 + lane];
                p.x = fminf(p.x, r.x); p.y = fminf(p.y, r.y); p.z = fminf(p.z, r.z);
                q.x = fmaxf(q.x, r.x); q.y = fmaxf(q.y, r.y); q.z = fmaxf(q.z, r.z);
            }
            const uint32_t lx = __reduce_min_sync(0xffffffffu, ord_key(p.x));
            const uint32_t ly = __reduce_min_sync(0xffffffffu, ord_key(p.y));
            const uint32_t lz = __reduce_min_sync(0xffffffffu, ord_key(p.z));
            const uint32_t hx = __reduce_max_sync(0xffffffffu, ord_key(q.x));
            const uint32_t hy = __reduce_max_sync(0xffffffffu, ord_key(q.y));
            const uint32_t hz = __reduce_max_sync(0xffffffffu, ord_key(q.z));
            if (lane == 0) {
                float* lo = nodes[j].c[side].lo;
                lo[0] = ord_float(lx); lo[1] = ord_float(ly); lo[2] = ord_float(lz);
                lo[3] = ord_float(hx); lo[4] = ord_float(hy); lo[5] = ord_float(hz);
            }
        }
    }
}

// Thread per compacted node: nodes whose two children are leaves start a
// climb; each climber writes its box into the parent's slot and the second
// arrival at a parent continues upwards.
__device__ __forceinline__ void refit_thread(Node* nodes, const uint32_t* __restrict__ parent, uint32_t* arrive,
                                             const uint32_t* __restrict__ nleaf, const MapHeader* __restrict__ hdr,
                                             uint32_t max_nodes, uint32_t t) {
    const uint32_t m = hdr->num_nodes;
    if (t >= m || t >= max_nodes) return;
    uint32_t id = 1 + t;
    if (nleaf[id] != 2) return;
    for (;;) {
        const float* s0 = nodes[id].c[0].lo;
        const float* s1 = nodes[id].c[1].lo;
        float box[6];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            box[a] = fminf(__ldcg(s0 + a), __ldcg(s1 + a));
            box[a + 3] = fmaxf(__ldcg(s0 + 3 + a), __ldcg(s1 + 3 + a));
        }
        uint32_t p, side;
        if (id == 1) { p = 0; side = 0; }
        else { const uint32_t ps = parent[id]; p = ps >> 1; side = ps & 1u; }
        float* dst = nodes[p].c[side].lo;
#pragma unroll
        for (int a = 0; a < 6; ++a) __stcg(dst + a, box[a]);
        if (p == 0) break;
        __threadfence();
        const uint32_t old = atomicAdd(&arrive[p], 1u);
        if (old != 1u) break;     // the sibling subtree is still being refitted
        __threadfence();
        id = p;
    }
}

__global__ void k_refit(Node* nodes, const uint32_t* __restrict__ parent, uint32_t* arrive,
                        const uint32_t* __restrict__ nleaf, const MapHeader* __restrict__ hdr, uint32_t max_nodes) {
    refit_thread(nodes, parent, arrive, nleaf, hdr, max_nodes, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void k_scale_flux(float4* pw, uint32_t n, float scale, MapHeader* hdr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        hdr->max_power = __fmul_rn(hdr->max_power, fabsf(scale));
        hdr->fix_scale = fix_scale_of(hdr->max_power);
    }
    if (i >= n) return;
    float4 w = pw[i];
    w.x = __fmul_rn(w.x, scale);
    w.y = __fmul_rn(w.y, scale);
    w.z = __fmul_rn(w.z, scale);
    pw[i] = w;
}

void scale_flux(float4* pw, uint32_t n, float scale, MapHeader* hdr, cudaStream_t st) {
    const uint32_t blocks = n ? (n + 255) / 256 : 1;
    k_scale_flux<<<blocks, 256, 0, st>>>(pw, n, scale, hdr);
}

// Everything after the sort: photons into tree order (unless the sort's last
// pass already moved them: gathered), radix tree, compaction into 64-byte
// nodes, refit.  keys/vals are the sorted (code, caller index) pairs; any
// code whose prefix separates groups (e.g. a map id in the top bits) yields
// one subtree per group.
// k_refit_wide_count is defined with the wide tree below.
__global__ void k_refit_wide_count(Node* nodes, const uint32_t* __restrict__ parent, uint32_t* arrive,
                                   const uint32_t* __restrict__ nleaf, const MapHeader* __restrict__ hdr,
                                   uint32_t max_nodes, uint32_t refit_blocks, uint32_t bound,
                                   uint32_t* __restrict__ wflag, uint32_t* __restrict__ wcnt,
                                   uint32_t* __restrict__ wfirst, uint32_t* scan, uint32_t* err);
__global__ void k_wide_emit(const Node* __restrict__ nodes, const uint32_t* __restrict__ rootmark,
                            const uint32_t* __restrict__ wflag, const uint32_t* __restrict__ wcnt,
                            const uint32_t* __restrict__ wfirst, const MapHeader* __restrict__ hdr, uint32_t bound,
                            ChildSlot* __restrict__ wchild, ChildSlot* __restrict__ wroot);

int build_from_sorted(const float4* in_pos, const float4* in_pow, uint32_t n, int format, uint32_t leaf_size,
                      const uint64_t* keys, const uint32_t* vals, float4* out_pos, float4* out_pow, uint32_t* inv,
                      Node* nodes, MapHeader* hdr, const BuildBuffers& bb, cudaStream_t st, bool gathered,
                      const WideBuffers* wide) {
    const uint32_t tb = 256;
    if (n > 0) {
        if (!gathered) k_gather<<<(n + tb - 1) / tb, tb, 0, st>>>(in_pos, in_pow, vals, n, format, out_pos, out_pow, inv);
        const int ng = gathered ? 0 : 1;
        if (n > 1) {
            const uint32_t ni = n - 1, gi = (ni + tb - 1) / tb;
            // the keep flags' exclusive scan (a single-pass scan with look-back inside
            // k_radix_tree measured 87 us against 46 + 13 us: one slow tile holds up
            // every later one, where separate kernels let blocks finish independently)
            k_radix_tree<<<gi, tb, 0, st>>>(keys, n, leaf_size, bb.kfirst, bb.klast, bb.ksplit, bb.kkeep);
            uint32_t* total = bb.scratch + sort_scratch_words(n);
            const int ns = exclusive_scan(bb.kkeep, bb.krank, ni, total + 1, total, st);
            k_emit<<<gi, tb, 0, st>>>(out_pos, n, leaf_size, bb.kfirst, bb.klast, bb.ksplit, bb.kkeep, bb.krank,
                                      total, nodes, bb.parent, bb.arrive, bb.nleaf, hdr);
            k_leaf_boxes<<<kLeafBoxBlocks, 256, 0, st>>>(out_pos, nodes, hdr);
            if (wide) {   // the single-map build: refit and the wide tree's counts in one launch
                const uint32_t wgrid = (ni + 255u) / 256u;
                cudaMemsetAsync(wide->scratch, 0, wide_scan_words(n) * sizeof(uint32_t), st);
                k_refit_wide_count<<<gi + wgrid, tb, 0, st>>>(nodes, bb.parent, bb.arrive, bb.nleaf, hdr, n, gi, ni,
                                                             wide->wflag, wide->wcnt, wide->wfirst, wide->scratch,
                                                             &hdr->errors);
                k_wide_emit<<<wgrid, 256, 0, st>>>(nodes, nullptr, wide->wflag, wide->wcnt, wide->wfirst, hdr, ni,
                                                   wide->wchild, wide->wroot);
                return ng + 6 + ns;
            }
            k_refit<<<gi, tb, 0, st>>>(nodes, bb.parent, bb.arrive, bb.nleaf, hdr, n);
            return ng + 5 + ns;
        }
    }
    k_emit<<<1, 32, 0, st>>>(out_pos, n, leaf_size, bb.kfirst, bb.klast, bb.ksplit, bb.kkeep, bb.krank, nullptr,
                             nodes, bb.parent, bb.arrive, bb.nleaf, hdr);
    return n > 0 ? 2 : 1;
}

int build_map(const float4* in_pos, const float4* in_pow, uint32_t n, int format, uint32_t leaf_size,
              float4* out_pos, float4* out_pow, uint32_t* inv, Node* nodes, MapHeader* hdr, const BuildBuffers& bb,
              const WideBuffers& wide, cudaStream_t st, cudaEvent_t sort_done) {
    int nl = 0;
    const uint32_t nb = (uint32_t)((n + kBoundsThreads - 1) / kBoundsThreads);
    const uint32_t bblocks = nb < 1 ? 1 : (nb > (uint32_t)kBoundsBlocksMax ? (uint32_t)kBoundsBlocksMax : nb);
    cudaMemsetAsync(&hdr->errors, 0, sizeof(uint32_t), st);
    cudaMemsetAsync(bb.partials + 8 * bblocks, 0, sizeof(uint32_t), st);
    k_bounds<<<bblocks, kBoundsThreads, 0, st>>>(in_pos, in_pow, n, reinterpret_cast<float*>(bb.partials), hdr);
    ++nl;
    uint64_t* keys[2] = {bb.keys[0], bb.keys[1]};
    uint32_t* vals[2] = {bb.vals[0], bb.vals[1]};
    int cur = 0;
    if (n > 0) {
        const uint32_t tb = 256;
        k_morton<<<(n + tb - 1) / tb, tb, 0, st>>>(in_pos, n, hdr, bb.keys[0], bb.vals[0]);
        ++nl;
        // the last pass moves the photons into tree order (n >= 2; one photon is not sorted)
        const SortGather g{in_pos, in_pow, format, out_pos, out_pow, inv};
        cur = radix_sort_pairs(keys, vals, n, kMortonBits, bb.scratch, st, &nl, n > 1 ? &g : nullptr);
    }
    if (sort_done) cudaEventRecord(sort_done, st);
    nl += build_from_sorted(in_pos, in_pow, n, format, leaf_size, keys[cur], vals[cur], out_pos, out_pow, inv, nodes,
                            hdr, bb, st, n > 1, &wide);
    if (n <= 1) nl += build_wide(n, nodes, bb.parent, nullptr, hdr, wide, st);   // the start slot only
    return nl;
}


// ---------------------------------------------------------------- wide tree --

__device__ __forceinline__ bool is_marked_root(const uint32_t* rootmark, uint32_t id) {
    return id == 1 || (rootmark && rootmark[id]);
}

// Warp-cooperative expansion of wide node `id`: the slots reached by expanding
// kWideLevels binary levels, in tree order (left to right), item i held by
// lane i.  A slot ends the expansion when it is a leaf, or an internal node
// at the last level or at a map's root (which becomes a wide child); empty
// slots are dropped.  Items are compacted level by level through `sbuf`
// (64 words of the warp's shared memory).  Returns the item count (<= 32).
constexpr uint32_t kItemPending = 0, kItemLeaf = 1, kItemWide = 2;

__device__ uint32_t wide_expand_warp(const Node* __restrict__ nodes, const uint32_t* __restrict__ rootmark,
                                     uint32_t id, uint32_t lane, uint32_t* sbuf, uint32_t& slot, uint32_t& state) {
    uint32_t count = 2;
    slot = 2u * id + lane;
    state = kItemPending;
    for (int lvl = 1; lvl <= kWideLevels; ++lvl) {
        uint32_t nout = 0, ref = kInvalid;
        if (lane < count) {
            nout = 1;
            if (state == kItemPending) {
                const ChildSlot& s = nodes[slot >> 1].c[slot & 1u];
                ref = s.ref;
                if (ref == kInvalid) nout = 0;
                else if (s.cnt > 0) state = kItemLeaf;
                else if (lvl == kWideLevels || is_marked_root(rootmark, ref)) state = kItemWide;
                else nout = 2;
            }
        }
        uint32_t x = nout;   // inclusive scan of the output counts
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if ((int)lane >= o) x += y;
        }
        const uint32_t at = x - nout, total = __shfl_sync(0xffffffffu, x, 31);
        if (nout == 1) {
            sbuf[at] = slot;
            sbuf[32 + at] = state;
        } else if (nout == 2) {
            sbuf[at] = 2u * ref;
            sbuf[at + 1] = 2u * ref + 1u;
            sbuf[32 + at] = kItemPending;
            sbuf[32 + at + 1] = kItemPending;
        }
        __syncwarp();
        count = total;
        if (lane < count) { slot = sbuf[lane]; state = sbuf[32 + lane]; }
        __syncwarp();
    }
    return count;
}

// Block of 8 warps per 256 consecutive compacted nodes, taken by ticket: each
// lane marks its node as wide when the node lies a multiple of kWideLevels
// below its root (node 1, or a node marked in rootmark), the warps expand
// their wide nodes to count the children, and the block's exclusive scan of
// the counts plus a decoupled look-back gives every wide node its first
// child slot (one launch for flags, counts and scan).  scan: [0] ticket, [1]
// total child slots (last tile), look-back words from word 2; cleared before.
__device__ __forceinline__ void wide_count_block(const Node* __restrict__ nodes, const uint32_t* __restrict__ parent,
                                                 const uint32_t* __restrict__ rootmark,
                                                 const MapHeader* __restrict__ hdr, uint32_t bound,
                                                 uint32_t* __restrict__ wflag, uint32_t* __restrict__ wcnt,
                                                 uint32_t* __restrict__ wfirst, uint32_t* scan, uint32_t* err) {
    __shared__ uint32_t s_buf[8][64];
    __shared__ uint32_t s_tile, s_warp[32];
    __shared__ uint64_t s_before;
    if (threadIdx.x == 0) s_tile = atomicAdd(&scan[0], 1u);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t t0 = s_tile * 256u + wib * 32u;
    const uint32_t m = hdr->num_nodes;
    const uint32_t t = t0 + lane;
    bool wide = false;
    if (t < m && t < bound) {
        uint32_t c = t + 1, d = 0;
        while (!is_marked_root(rootmark, c) && d < 4096) { c = parent[c] >> 1; ++d; }
        wide = d % kWideLevels == 0;
    }
    uint32_t mine = 0;
    uint32_t todo = __ballot_sync(0xffffffffu, wide);
    while (todo) {
        const uint32_t b = __ffs(todo) - 1;
        todo &= todo - 1;
        uint32_t slot, state;
        const uint32_t c = wide_expand_warp(nodes, rootmark, t0 + b + 1u, lane, s_buf[wib], slot, state);
        if (lane == b) mine = c;
    }
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(mine, s_warp, total);
    if (threadIdx.x < 32) {
        const uint64_t b = warp_lookback_exclusive(reinterpret_cast<uint64_t*>(scan + 2), s_tile, total, err);
        if (threadIdx.x == 0) s_before = b;
    }
    __syncthreads();
    if (t < bound) {
        wflag[t] = wide ? 1u : 0u;
        wcnt[t] = mine;
        wfirst[t] = (uint32_t)s_before + ex;
    }
    if (threadIdx.x == 0 && s_tile + 1 == (bound + 255u) / 256u) scan[1] = (uint32_t)s_before + total;
}

__global__ void __launch_bounds__(256) k_wide_count(const Node* __restrict__ nodes, const uint32_t* __restrict__ parent,
                                                     const uint32_t* __restrict__ rootmark,
                                                     const MapHeader* __restrict__ hdr, uint32_t bound,
                                                     uint32_t* __restrict__ wflag, uint32_t* __restrict__ wcnt,
                                                     uint32_t* __restrict__ wfirst, uint32_t* scan, uint32_t* err) {
    wide_count_block(nodes, parent, rootmark, hdr, bound, wflag, wcnt, wfirst, scan, err);
}

// The refit and the wide tree's counts in one launch: they are independent
// (the counts read only the tree's structure, which k_emit wrote; the refit
// writes only boxes), and both are latency-bound walks along root-to-leaf
// paths, so blocks [0, refit_blocks) climb while the others count.  The
// counting blocks take their tiles by ticket and wait only on each other.
__global__ void __launch_bounds__(256) k_refit_wide_count(Node* nodes, const uint32_t* __restrict__ parent,
                                                           uint32_t* arrive, const uint32_t* __restrict__ nleaf,
                                                           const MapHeader* __restrict__ hdr, uint32_t max_nodes,
                                                           uint32_t refit_blocks, uint32_t bound,
                                                           uint32_t* __restrict__ wflag, uint32_t* __restrict__ wcnt,
                                                           uint32_t* __restrict__ wfirst, uint32_t* scan,
                                                           uint32_t* err) {
    if (blockIdx.x < refit_blocks) {
        refit_thread(nodes, parent, arrive, nleaf, hdr, max_nodes, blockIdx.x * blockDim.x + threadIdx.x);
        return;
    }
    wide_count_block(nodes, parent, nullptr, hdr, bound, wflag, wcnt, wfirst, scan, err);
}

// Warp per 32 consecutive compacted nodes: every wide node's child slots;
// thread 0 of block 0 also writes the traversal's start slot (the
// super-root's slot, pointing at the root wide node).
__global__ void k_wide_emit(const Node* __restrict__ nodes, const uint32_t* __restrict__ rootmark,
                            const uint32_t* __restrict__ wflag, const uint32_t* __restrict__ wcnt,
                            const uint32_t* __restrict__ wfirst, const MapHeader* __restrict__ hdr, uint32_t bound,
                            ChildSlot* __restrict__ wchild, ChildSlot* __restrict__ wroot) {
    __shared__ uint32_t s_buf[8][64];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ChildSlot s = nodes[0].c[0];
        if (s.ref != kInvalid && s.cnt == 0) {
            s.ref = wfirst[0];
            s.cnt = kWideFlag | wcnt[0];
        }
        *wroot = s;
    }
    const uint32_t t0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u;
    if (t0 >= bound) return;
    const uint32_t m = hdr->num_nodes;
    const uint32_t t = t0 + lane;
    uint32_t todo = __ballot_sync(0xffffffffu, t < m && t < bound && wflag[t]);
    while (todo) {
        const uint32_t b = __ffs(todo) - 1;
        todo &= todo - 1;
        uint32_t slot, state;
        const uint32_t tb = t0 + b;
        const uint32_t c = wide_expand_warp(nodes, rootmark, tb + 1u, lane, s_buf[wib], slot, state);
        if (lane < c) {
            ChildSlot s = nodes[slot >> 1].c[slot & 1u];
            if (state == kItemWide) {
                const uint32_t r = s.ref;
                s.ref = wfirst[r - 1];
                s.cnt = kWideFlag | wcnt[r - 1];
            }
            wchild[wfirst[tb] + lane] = s;
        }
    }
}

int build_wide(uint32_t n, const Node* nodes, const uint32_t* parent, const uint32_t* rootmark, MapHeader* hdr,
               const WideBuffers& wb, cudaStream_t st) {
    const uint32_t bound = n > 1 ? n - 1 : 1;   // internal nodes are at most n - 1
    const uint32_t wgrid = (bound + 32u * 8u - 1u) / (32u * 8u);   // 8 warps per block, 32 nodes per warp
    if (n > 1) {
        cudaMemsetAsync(wb.scratch, 0, wide_scan_words(n) * sizeof(uint32_t), st);
        k_wide_count<<<wgrid, 256, 0, st>>>(nodes, parent, rootmark, hdr, bound, wb.wflag, wb.wcnt, wb.wfirst,
                                            wb.scratch, &hdr->errors);
    }
    k_wide_emit<<<n > 1 ? wgrid : 1, 256, 0, st>>>(nodes, rootmark, wb.wflag, wb.wcnt, wb.wfirst, hdr,
                                                  n > 1 ? bound : 0, wb.wchild, wb.wroot);
    return n > 1 ? 2 : 1;
}

}  // namespace pm
