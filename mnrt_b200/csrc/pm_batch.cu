// pm_batch.cu -- many photon maps built and queried together.
//
// The reference builds and queries one map per call (PhotonMap::BuildMap,
// PhotonMap::GatherFor); the batch form has no counterpart there.  Photons of
// all maps sit in one array (map i owns [ph_off_i, ph_off_i + n_i)), and so do
// the queries.  The build sorts every photon once by the 64-bit key
//   (map id << 39) | 39-bit Morton code in the map's own cubic cell,
// so one radix tree holds every map: the map id bits split first, and the
// node whose range is exactly a map's photons roots that map's subtree
// (k_batch_roots).  The query sorts all queries by (map id << 30) | 30-bit
// Hilbert index in the map's cell and runs one persistent launch over them
// (k_knn_group<32, *, true>), each query reading its map's root slot and
// parameters.
#include "pm_internal.h"

namespace pm {

namespace {

// Order-preserving map of floats to unsigned integers (min/max by integer
// atomics, exact and independent of the order of arrival).
__device__ __forceinline__ uint32_t f2ord(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Map owning element i of a batch with offsets off[0..m] (off[m] = total).
__device__ __forceinline__ uint32_t map_of(const uint32_t* __restrict__ off, uint32_t m, uint32_t i) {
    uint32_t lo = 0, hi = m;   // off[lo] <= i < off[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// acc: per map 8 words: ord(min x, y, z), ord(max x, y, z), ord(max flux), error flag.
__global__ void k_batch_bounds(const float4* __restrict__ pos, const float4* __restrict__ pw,
                               const uint32_t* __restrict__ off, uint32_t m, uint32_t n, uint32_t* __restrict__ acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    uint32_t map = 0;
    float v[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, 0.0f};
    uint32_t bad = 0;
    if (valid) {
        map = map_of(off, m, i);
        const float4 p = pos[i], w = pw[i];
        if (isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
            v[0] = v[3] = p.x; v[1] = v[4] = p.y; v[2] = v[5] = p.z;
            v[6] = fmaxf(fmaxf(fabsf(w.x), fabsf(w.y)), fabsf(w.z));
        } else {
            bad = 1;
        }
    }
    const uint32_t first = __shfl_sync(0xffffffffu, map, 0);
    const bool uniform = __all_sync(0xffffffffu, !valid || map == first) && __any_sync(0xffffffffu, valid);
    if (uniform) {   // the common case: the warp lies inside one map
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            for (int a = 0; a < 3; ++a) {
                v[a] = fminf(v[a], __shfl_xor_sync(0xffffffffu, v[a], o));
                v[a + 3] = fmaxf(v[a + 3], __shfl_xor_sync(0xffffffffu, v[a + 3], o));
            }
            v[6] = fmaxf(v[6], __shfl_xor_sync(0xffffffffu, v[6], o));
        }
        bad = __any_sync(0xffffffffu, bad) ? 1u : 0u;
        if ((threadIdx.x & 31u) != 0) return;
        map = first;
    } else if (!valid) {
        return;
    }
    uint32_t* a = acc + 8 * (size_t)map;
    if (v[0] <= v[3]) {   // at least one finite photon
        for (int c = 0; c < 3; ++c) { atomicMin(a + c, f2ord(v[c])); atomicMax(a + 3 + c, f2ord(v[c + 3])); }
    }
    atomicMax(a + 6, f2ord(v[6]));
    if (bad) atomicOr(a + 7, 1u);
}

__global__ void k_batch_acc_init(uint32_t* __restrict__ acc, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t* a = acc + 8 * (size_t)i;
    for (int c = 0; c < 3; ++c) { a[c] = 0xffffffffu; a[3 + c] = 0u; }
    a[6] = f2ord(0.0f);
    a[7] = 0u;
}

__global__ void k_batch_geom(const uint32_t* __restrict__ acc, uint32_t m, BatchGeom* __restrict__ geom,
                             MapHeader* __restrict__ hdr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t* a = acc + 8 * (size_t)i;
    BatchGeom g;
    float hi[3];
    const bool any = a[0] != 0xffffffffu;
    for (int c = 0; c < 3; ++c) {
        g.lo[c] = any ? ord2f(a[c]) : 0.0f;
        hi[c] = any ? ord2f(a[3 + c]) : 0.0f;
    }
    const float ext = fmaxf(fmaxf(__fsub_rn(hi[0], g.lo[0]), __fsub_rn(hi[1], g.lo[1])), __fsub_rn(hi[2], g.lo[2]));
    g.mscale = (ext > 0.0f && isfinite(ext)) ? __fdiv_rn(65536.0f, ext) : 0.0f;
    g.max_power = ord2f(a[6]);
    g.fix_scale = fix_scale_of(g.max_power);
    g.pad[0] = g.pad[1] = 0;
    g.root.lo[0] = g.root.lo[1] = g.root.lo[2] = INFINITY;
    g.root.hi[0] = g.root.hi[1] = g.root.hi[2] = -INFINITY;
    g.root.ref = kInvalid;
    g.root.cnt = 0;
    geom[i] = g;
    if (a[7]) atomicOr(&hdr->errors, kErrNonFinite);
}

// Query keys: map id above bit 30, Hilbert index in the map's cell (the
// processing order only; 30 + map-id bits sort in fewer passes than the
// photons' 39-bit codes).
__global__ void k_batch_query_keys(const float4* __restrict__ pts, const uint32_t* __restrict__ off, uint32_t m,
                                   uint32_t n, const BatchGeom* __restrict__ geom, uint64_t* __restrict__ keys,
                                   uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t map = map_of(off, m, i);
    const BatchGeom& g = geom[map];
    const float4 p = pts[i];
    keys[i] = ((uint64_t)map << kBatchQueryMapShift) | hilbert30(p.x, p.y, p.z, g.lo, g.mscale);
    vals[i] = i;
}

// Photon keys: map id above bit kMortonBits, Morton code in the map's cell.
__global__ void k_batch_keys(const float4* __restrict__ pts, const uint32_t* __restrict__ off, uint32_t m, uint32_t n,
                             const BatchGeom* __restrict__ geom, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t map = map_of(off, m, i);
    const BatchGeom& g = geom[map];
    const float4 p = pts[i];
    keys[i] = ((uint64_t)map << kMortonBits) | morton39(p.x, p.y, p.z, g.lo, g.mscale);
    vals[i] = i;
}

__device__ __forceinline__ void slot_box(const float4* __restrict__ pos, uint32_t first, uint32_t cnt, ChildSlot& s) {
    float lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY, hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY;
    for (uint32_t k = 0; k < cnt; ++k) {
        const float4 p = pos[first + k];
        lo0 = fminf(lo0, p.x); lo1 = fminf(lo1, p.y); lo2 = fminf(lo2, p.z);
        hi0 = fmaxf(hi0, p.x); hi1 = fmaxf(hi1, p.y); hi2 = fmaxf(hi2, p.z);
    }
    s.lo[0] = lo0; s.lo[1] = lo1; s.lo[2] = lo2;
    s.hi[0] = hi0; s.hi[1] = hi1; s.hi[2] = hi2;
}

// Root slot of every map: a leaf when the map holds at most leaf_size
// photons, else a copy of the slot that references the radix-tree node whose
// range is exactly the map's photons (that node's index is one end of its
// range, so it is node s or node e - 1).
__global__ void k_batch_roots(const uint32_t* __restrict__ off, uint32_t m, uint32_t n, uint32_t leaf_size,
                              const float4* __restrict__ pos, const Node* __restrict__ nodes,
                              const uint32_t* __restrict__ kfirst, const uint32_t* __restrict__ klast,
                              const uint32_t* __restrict__ krank, const uint32_t* __restrict__ parent,
                              BatchGeom* __restrict__ geom) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t s = off[i], e = off[i + 1];
    ChildSlot slot = geom[i].root;   // empty
    if (e > s && e - s <= leaf_size) {
        slot_box(pos, s, e - s, slot);
        slot.ref = s;
        slot.cnt = e - s;
    } else if (e > s) {
        uint32_t r = kInvalid;
        if (s < n - 1 && kfirst[s] == s && klast[s] == e - 1) r = s;
        else if (e - 1 < n - 1 && kfirst[e - 1] == s && klast[e - 1] == e - 1) r = e - 1;
        if (r != kInvalid) {
            const uint32_t id = 1 + krank[r];
            if (id == 1) {
                slot = nodes[0].c[0];
            } else {
                const uint32_t ps = parent[id];
                slot = nodes[ps >> 1].c[ps & 1u];
            }
        }
    }
    geom[i].root = slot;
}

// Marks every map's root node (internal) so that the wide tree starts a wide
// node there.
__global__ void k_batch_rootmark(const BatchGeom* __restrict__ geom, uint32_t m, uint32_t* __restrict__ rootmark) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const ChildSlot& s = geom[i].root;
    if (s.ref != kInvalid && s.cnt == 0) rootmark[s.ref] = 1u;
}

// Every map's start slot in the wide tree.
__global__ void k_batch_wroots(const uint32_t* __restrict__ wcnt, const uint32_t* __restrict__ wfirst, uint32_t m,
                               BatchGeom* __restrict__ geom) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    ChildSlot s = geom[i].root;
    if (s.ref != kInvalid && s.cnt == 0) {
        const uint32_t t = s.ref - 1;
        s.ref = wfirst[t];
        s.cnt = kWideFlag | wcnt[t];
    }
    geom[i].wroot = s;
}

}  // namespace

int batch_wide(uint32_t n, uint32_t m, const Node* nodes, const uint32_t* parent, MapHeader* hdr, uint32_t* rootmark,
               const WideBuffers& wb, BatchGeom* geom, cudaStream_t st) {
    cudaMemsetAsync(rootmark, 0, (size_t)(n + 1) * sizeof(uint32_t), st);
    k_batch_rootmark<<<(m + 127) / 128, 128, 0, st>>>(geom, m, rootmark);
    int nl = 1 + build_wide(n, nodes, parent, rootmark, hdr, wb, st);
    k_batch_wroots<<<(m + 127) / 128, 128, 0, st>>>(wb.wcnt, wb.wfirst, m, geom);
    return nl + 1;
}

int batch_bounds_and_keys(const float4* pos, const float4* pw, const uint32_t* ph_off, uint32_t m, uint32_t n,
                          uint32_t* acc, BatchGeom* geom, MapHeader* hdr, uint64_t* keys, uint32_t* vals,
                          cudaStream_t st) {
    int nl = 0;
    cudaMemsetAsync(&hdr->errors, 0, sizeof(uint32_t), st);
    k_batch_acc_init<<<(m + 127) / 128, 128, 0, st>>>(acc, m);
    ++nl;
    if (n > 0) {
        k_batch_bounds<<<(n + 255) / 256, 256, 0, st>>>(pos, pw, ph_off, m, n, acc);
        ++nl;
    }
    k_batch_geom<<<(m + 127) / 128, 128, 0, st>>>(acc, m, geom, hdr);
    ++nl;
    if (n > 0) {
        k_batch_keys<<<(n + 255) / 256, 256, 0, st>>>(pos, ph_off, m, n, geom, keys, vals);
        ++nl;
    }
    return nl;
}

int batch_query_keys(const float4* qpos, const uint32_t* q_off, uint32_t m, uint32_t nq, const BatchGeom* geom,
                     uint64_t* keys, uint32_t* vals, cudaStream_t st) {
    if (!nq) return 0;
    k_batch_query_keys<<<(nq + 255) / 256, 256, 0, st>>>(qpos, q_off, m, nq, geom, keys, vals);
    return 1;
}

int batch_roots(const uint32_t* ph_off, uint32_t m, uint32_t n, uint32_t leaf_size, const float4* pos,
                const Node* nodes, const BuildBuffers& bb, BatchGeom* geom, cudaStream_t st) {
    k_batch_roots<<<(m + 127) / 128, 128, 0, st>>>(ph_off, m, n, leaf_size, pos, nodes, bb.kfirst, bb.klast, bb.krank,
                                                    bb.parent, geom);
    return 1;
}

int map_id_bits(uint32_t m) {
    int b = 0;
    while (b < 16 && (1u << b) < m) ++b;
    return b;
}

}  // namespace pm
