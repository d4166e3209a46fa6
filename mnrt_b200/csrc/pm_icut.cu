// pm_icut.cu -- illumination cuts over the photon tree.
//
// An illumination cut (Wang et al. 2009, as the reference builds it in
// GPU/illumcut.cu, PhotonMap.cpp:287-452 and GPU/photon_knn.cu:338-433,
// 598-716) is a set of tree nodes with a node on every root-to-leaf path.
// Irradiance is estimated once at each cut node's centre; a final-gather
// query then interpolates the cut nodes near it instead of searching
// photons.  The engine's tree nodes are its child slots: slot 2j + side of
// internal node j, slot 0 the root (slot 1 is always empty).
//
//   1. per slot: level (root 0), photon range, box centre and largest side
//      (illumcut.cu:108-119; PhotonMap.cpp:366-367)
//   2. per slot normal: the caller's (the reference takes it from the scene
//      geometry, PhotonMap.cpp:339-364) or, without one, the normalised sum
//      of the photons' reversed incident directions (slots under 5,000
//      photons; larger ones get none)
//   3. photon-sum estimate E~ = sum(front * flux) / side^2 over slots with
//      0 < photons < 5,000 and a normal (illumcut.cu:151-209)
//   4. coarse cut: every leaf (ICutUseLeafs), or the slots whose E~ reaches
//      E_min in every component (E_min = mean of the nonzero E~ on level
//      level_emin), without parents whose children are both or neither
//      marked, made a cut top-down (illumcut.cu:222-440, 627-680)
//   5. irradiance at every slot centre with the slot's normal: the engine's
//      query (exact kNN, or PM_MODE_ZHOU_COMPAT for the reference's radius
//      pipeline; PhotonMap.cpp:371-384, photon_knn.cu:686-716)
//   6. final cut: refine_iters rounds over a work set that starts as the
//      coarse cut; a work slot joins the cut when it is a leaf or
//      |E~ - E| < accuracy * E in every component, otherwise its children
//      become work; what is left joins the cut (illumcut.cu:488-519,
//      PhotonMap.cpp:387-452)
//   7. interpolation at a query q with normal n: every cut slot (or leaf)
//      reached through slots whose box lies within R of q contributes
//      w = (1 - t^2) * max(0, n_slot . n), t = |centre - q| / side <= 1;
//      E(q) = sum(w E) / sum(w) (photon_knn.cu:338-433, 598-660).  A cut
//      slot's weight is zero unless q lies in the cube of half-width side
//      about its centre, so each slot also carries an influence box: the
//      union of those cubes (slightly widened) over the cut slots where
//      interpolation below it stops.  The traversal skips slots whose
//      influence box misses q, which removes only zero terms.
//
// Determinism: sums over a slot's photons run lane-strided over one warp and
// then down a fixed xor butterfly; the level mean of step 4 is an exact
// 64-bit fixed-point sum; the refinement works on 0/1 flags (a slot both
// finished and re-added by its parent stays work: adding wins).
#include "pm_internal.h"

namespace pm {

namespace {

constexpr uint32_t kIcutPhotonLimit = 5000;   // ICUT_PHOTONLIMIT, illumcut.cu:74
constexpr int kIcutMaxDepth = 4096;           // bound of every walk up or down the tree
constexpr int kIcutStack = 128;               // interpolation traversal stack per query

__device__ __forceinline__ void slot_load(const Node* __restrict__ nodes, uint32_t sid, float* lo, float* hi,
                                          uint32_t& ref, uint32_t& cnt) {
    const float4* p = reinterpret_cast<const float4*>(&nodes[sid >> 1].c[sid & 1u]);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    lo[0] = a.x; lo[1] = a.y; lo[2] = a.z; hi[0] = a.w;
    hi[1] = b.x; hi[2] = b.y; ref = __float_as_uint(b.z); cnt = __float_as_uint(b.w);
}

__device__ __forceinline__ uint32_t slot_ref(const Node* __restrict__ nodes, uint32_t sid) {
    return nodes[sid >> 1].c[sid & 1u].ref;
}
__device__ __forceinline__ uint32_t slot_cnt(const Node* __restrict__ nodes, uint32_t sid) {
    return nodes[sid >> 1].c[sid & 1u].cnt;
}

__device__ __forceinline__ float dot3_rn(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// Sum over the warp down the fixed butterfly 16, 8, 4, 2, 1 (every lane ends
// with the same bits: a + b == b + a).
__device__ __forceinline__ float warp_sum_fixed(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Node j -> the slot that references it (node 1, the root node, is
// referenced by slot 0).
__global__ void k_icut_parents(const Node* __restrict__ nodes, uint32_t m, uint32_t* __restrict__ pslot) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > m) return;
    if (j == 0) {
        if (m > 0) pslot[1] = 0u;
        return;
    }
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const ChildSlot& s = nodes[j].c[side];
        if (s.ref != kInvalid && s.cnt == 0) pslot[s.ref] = 2u * j + (uint32_t)side;
    }
}

// Per slot: level, photon range [first, end), box centre (xyz) and largest
// box side (w).  Empty slots get level kInvalid and a zero record.
__global__ void k_icut_slots(const Node* __restrict__ nodes, uint32_t nslots, const uint32_t* __restrict__ pslot,
                             uint32_t* __restrict__ level, uint2* __restrict__ range, float4* __restrict__ center,
                             MapHeader* hdr) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    float lo[3], hi[3];
    uint32_t ref, cnt;
    slot_load(nodes, s, lo, hi, ref, cnt);
    if (ref == kInvalid) {
        level[s] = kInvalid;
        range[s] = make_uint2(0u, 0u);
        center[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    bool lost = false;   // a walk longer than any valid tree
    uint32_t lvl = 0, t = s;
    while (t > 1u) {
        if (lvl == (uint32_t)kIcutMaxDepth) { lost = true; break; }
        t = pslot[t >> 1];
        ++lvl;
    }
    uint32_t first = ref, end = ref + cnt;
    if (cnt == 0) {
        bool done0 = false, done1 = false;
        uint32_t j = ref;
        for (int g = 0; g < kIcutMaxDepth && !done0; ++g) {
            const ChildSlot& c = nodes[j].c[0];
            if (c.cnt > 0) { first = c.ref; done0 = true; }
            else j = c.ref;
        }
        j = ref;
        for (int g = 0; g < kIcutMaxDepth && !done1; ++g) {
            const ChildSlot& c = nodes[j].c[1];
            if (c.cnt > 0) { end = c.ref + c.cnt; done1 = true; }
            else j = c.ref;
        }
        lost = lost || !done0 || !done1;
    }
    if (lost) {
        atomicOr(&hdr->errors, kErrStack);
        first = end = 0;
    }
    level[s] = lvl;
    range[s] = make_uint2(first, end);
    float c[3], e[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e[a] = __fsub_rn(hi[a], lo[a]);
        c[a] = __fadd_rn(lo[a], __fmul_rn(0.5f, e[a]));
    }
    center[s] = make_float4(c[0], c[1], c[2], fmaxf(e[0], fmaxf(e[1], e[2])));
}

// Caller normals: xyz kept, w cleared.
__global__ void k_icut_copy_normals(const float4* __restrict__ in, uint32_t nslots, float4* __restrict__ out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const float4 v = in[s];
    out[s] = make_float4(v.x, v.y, v.z, 0.0f);
}

// Warp per slot: normalised sum of -d / |d| over the slot's photons (d = the
// decoded incident direction), for slots of fewer than kIcutPhotonLimit photons.
__global__ void k_icut_normals(const float4* __restrict__ pw, uint32_t nslots, const uint2* __restrict__ range,
                               float4* __restrict__ normal) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (s >= nslots) return;
    const uint2 r = range[s];
    const uint32_t count = r.y - r.x;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    if (count > 0 && count < kIcutPhotonLimit) {
        for (uint32_t i = r.x + lane; i < r.y; i += 32u) {
            float x, y, z;
            oct_decode(__float_as_uint(__ldg(&pw[i].w)), x, y, z);
            const float len = __fsqrt_rn(dot3_rn(x, y, z, x, y, z));
            if (len > 0.0f) {
                sx = __fsub_rn(sx, __fdiv_rn(x, len));
                sy = __fsub_rn(sy, __fdiv_rn(y, len));
                sz = __fsub_rn(sz, __fdiv_rn(z, len));
            }
        }
    }
    sx = warp_sum_fixed(sx);
    sy = warp_sum_fixed(sy);
    sz = warp_sum_fixed(sz);
    if (lane != 0) return;
    const float l = __fsqrt_rn(dot3_rn(sx, sy, sz, sx, sy, sz));
    normal[s] = l > 0.0f ? make_float4(__fdiv_rn(sx, l), __fdiv_rn(sy, l), __fdiv_rn(sz, l), 0.0f)
                         : make_float4(0.f, 0.f, 0.f, 0.f);
}

// Warp per slot: E~ = sum(front * flux) / side^2 (illumcut.cu:151-209).
__global__ void k_icut_estimate(const float4* __restrict__ pw, uint32_t nslots, const uint2* __restrict__ range,
                                const float4* __restrict__ center, const float4* __restrict__ normal,
                                float4* __restrict__ est) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (s >= nslots) return;
    const uint2 r = range[s];
    const uint32_t count = r.y - r.x;
    const float4 n = normal[s];
    const bool eval = count > 0 && count < kIcutPhotonLimit && dot3_rn(n.x, n.y, n.z, n.x, n.y, n.z) > 0.0f;
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (eval) {
        for (uint32_t i = r.x + lane; i < r.y; i += 32u) {
            const float4 w = __ldg(pw + i);
            if (front_rn(n.x, n.y, n.z, __float_as_uint(w.w))) {
                ax = __fadd_rn(ax, w.x);
                ay = __fadd_rn(ay, w.y);
                az = __fadd_rn(az, w.z);
            }
        }
    }
    ax = warp_sum_fixed(ax);
    ay = warp_sum_fixed(ay);
    az = warp_sum_fixed(az);
    if (lane != 0) return;
    const float side = center[s].w;
    if (!eval || !(side > 0.0f)) {
        est[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float a2 = __fmul_rn(side, side);
    est[s] = make_float4(__fdiv_rn(ax, a2), __fdiv_rn(ay, a2), __fdiv_rn(az, a2), 0.0f);
}

__device__ __forceinline__ bool icut_on_level(const uint32_t* level, const float4* est, uint32_t s, uint32_t L,
                                              float4& e) {
    if (level[s] != L) return false;
    e = est[s];
    return !(e.x == 0.0f && e.y == 0.0f && e.z == 0.0f);
}

// Level statistics, pass 1: largest |E~| per component and the slot count
// (acc[0..2] = float bits of the maxima, acc[6] = count).
__global__ void k_icut_level_max(const uint32_t* __restrict__ level, const float4* __restrict__ est, uint32_t nslots,
                                 uint32_t L, unsigned long long* acc) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    float4 e;
    if (s >= nslots || !icut_on_level(level, est, s, L, e)) return;
    atomicMax(reinterpret_cast<unsigned int*>(acc + 0), __float_as_uint(fabsf(e.x)));
    atomicMax(reinterpret_cast<unsigned int*>(acc + 1), __float_as_uint(fabsf(e.y)));
    atomicMax(reinterpret_cast<unsigned int*>(acc + 2), __float_as_uint(fabsf(e.z)));
    atomicAdd(acc + 6, 1ull);
}

__device__ __forceinline__ double icut_fix_scale(const unsigned long long* acc, int c) {
    const float mx = __uint_as_float(*reinterpret_cast<const unsigned int*>(acc + c));
    return mx > 0.0f ? __ddiv_rn(1099511627776.0, (double)mx) : 0.0;   // 2^40 / max
}

// Pass 2: exact fixed-point sums (acc[3..5], two's complement).
__global__ void k_icut_level_sum(const uint32_t* __restrict__ level, const float4* __restrict__ est, uint32_t nslots,
                                 uint32_t L, unsigned long long* acc) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    float4 e;
    if (s >= nslots || !icut_on_level(level, est, s, L, e)) return;
    const float v[3] = {e.x, e.y, e.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const long long t = __double2ll_rn(__dmul_rn((double)v[c], icut_fix_scale(acc, c)));
        atomicAdd(acc + 3 + c, (unsigned long long)t);
    }
}

// E_min component c: the mean of the level's nonzero estimates (+inf when the
// level has none, so nothing is marked by it).
__device__ __forceinline__ float icut_emin(const unsigned long long* acc, int c) {
    const unsigned long long cnt = acc[6];
    if (cnt == 0) return INFINITY;
    const double scale = icut_fix_scale(acc, c);
    if (scale == 0.0) return 0.0f;
    const double sum = (double)(long long)acc[3 + c];
    return __double2float_rn(__ddiv_rn(__ddiv_rn(sum, scale), (double)cnt));
}

// Marks by E_min (illumcut.cu:318-334).
__global__ void k_icut_mark0(const uint32_t* __restrict__ level, const float4* __restrict__ est, uint32_t nslots,
                             const unsigned long long* __restrict__ acc, uint32_t* __restrict__ mark0) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const float ex = icut_emin(acc, 0), ey = icut_emin(acc, 1), ez = icut_emin(acc, 2);
    const float4 e = est[s];
    mark0[s] = (level[s] != kInvalid && e.x >= ex && e.y >= ey && e.z >= ez) ? 1u : 0u;
}

// Unmarks internal slots whose children are both or neither marked
// (illumcut.cu:352-370).
__global__ void k_icut_remove_parents(const Node* __restrict__ nodes, uint32_t nslots,
                                      const uint32_t* __restrict__ mark0, uint32_t* __restrict__ mark1) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    uint32_t mk = mark0[s];
    const uint32_t ref = slot_ref(nodes, s);
    if (mk && ref != kInvalid && slot_cnt(nodes, s) == 0) {
        const uint32_t a = mark0[2u * ref], b = mark0[2u * ref + 1u];
        if (a == b) mk = 0u;
    }
    mark1[s] = mk;
}

// The top-down pass of illumcut.cu:384-440 in closed form.  With m the marks
// above, cov(s) = OR of m over the path from s up to, but not including, the
// root.  Final mark: the root keeps m (a root leaf is marked); another
// internal slot keeps m(s) when its parent is uncovered; a leaf is marked
// exactly when its parent is uncovered.
__global__ void k_icut_cover(const Node* __restrict__ nodes, uint32_t nslots, const uint32_t* __restrict__ pslot,
                             const uint32_t* __restrict__ mark1, uint32_t* __restrict__ coarse) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const uint32_t ref = slot_ref(nodes, s);
    if (ref == kInvalid) { coarse[s] = 0u; return; }
    const bool leaf = slot_cnt(nodes, s) > 0;
    if (s == 0) { coarse[s] = leaf ? 1u : mark1[0]; return; }
    bool cov = false;
    uint32_t p = pslot[s >> 1];
    for (int g = 0; g < kIcutMaxDepth && p != 0u; ++g) {
        cov = cov || mark1[p] != 0u;
        p = pslot[p >> 1];
    }
    coarse[s] = leaf ? (cov ? 0u : 1u) : ((mark1[s] && !cov) ? 1u : 0u);
}

__global__ void k_icut_leaves(const Node* __restrict__ nodes, uint32_t nslots, uint32_t* __restrict__ coarse) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    coarse[s] = (slot_ref(nodes, s) != kInvalid && slot_cnt(nodes, s) > 0) ? 1u : 0u;
}

// One refinement round (illumcut.cu:488-519): work slots that are leaves or
// accurate enough join the cut, the others hand their work to their children.
__global__ void k_icut_refine(const Node* __restrict__ nodes, uint32_t nslots, const float4* __restrict__ est,
                              const float4* __restrict__ exact, float accuracy, const uint32_t* __restrict__ win,
                              uint32_t* __restrict__ wout, uint32_t* __restrict__ fin) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots || !win[s]) return;
    const uint32_t ref = slot_ref(nodes, s);
    if (ref == kInvalid) return;
    bool ok = slot_cnt(nodes, s) > 0;
    if (!ok) {
        const float4 a = est[s], b = exact[s];
        ok = fabsf(__fsub_rn(a.x, b.x)) < __fmul_rn(accuracy, b.x) &&
             fabsf(__fsub_rn(a.y, b.y)) < __fmul_rn(accuracy, b.y) &&
             fabsf(__fsub_rn(a.z, b.z)) < __fmul_rn(accuracy, b.z);
    }
    if (ok) {
        fin[s] = 1u;
    } else {
        wout[2u * ref] = 1u;
        wout[2u * ref + 1u] = 1u;
    }
}

__global__ void k_icut_finalize(uint32_t nslots, const uint32_t* __restrict__ work, uint32_t* __restrict__ fin) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslots && work[s]) fin[s] = 1u;
}

// Thread per slot: whether interpolation stops here (a cut slot or a leaf
// with no cut slot above it), and the slot's own influence box: for a
// stopping slot that can carry weight (a normal and a side) the cube
// [c - h, c + h], h = side widened by 0.1 % plus a few units in the last place
// of the coordinates; otherwise empty.  lo.w = 1 marks a stopping slot.
__global__ void k_icut_ibox_own(const Node* __restrict__ nodes, uint32_t nslots, const uint32_t* __restrict__ pslot,
                                const uint32_t* __restrict__ fin, const float4* __restrict__ center,
                                const float4* __restrict__ normal, float4* __restrict__ ibox) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const uint32_t ref = slot_ref(nodes, s);
    bool stop = ref != kInvalid && (fin[s] != 0u || slot_cnt(nodes, s) > 0);
    if (stop && s > 1u) {   // reachable only without a cut slot above it
        uint32_t p = pslot[s >> 1];
        for (int g = 0; g < kIcutMaxDepth; ++g) {
            if (fin[p]) { stop = false; break; }
            if (p == 0u) break;
            p = pslot[p >> 1];
        }
    }
    float4 lo = make_float4(INFINITY, INFINITY, INFINITY, stop ? 1.0f : 0.0f);
    float4 hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
    if (stop) {
        const float4 c = center[s];
        const float4 n = normal[s];
        if (c.w > 0.0f && dot3_rn(n.x, n.y, n.z, n.x, n.y, n.z) != 0.0f) {
            const float mag = __fadd_rn(__fadd_rn(__fadd_rn(fabsf(c.x), fabsf(c.y)), fabsf(c.z)), c.w);
            const float h = __fadd_rn(__fmul_rn(c.w, 1.001f), __fmul_rn(mag, 3.814697265625e-06f));   // + mag * 2^-18
            lo = make_float4(__fsub_rn(c.x, h), __fsub_rn(c.y, h), __fsub_rn(c.z, h), 1.0f);
            hi = make_float4(__fadd_rn(c.x, h), __fadd_rn(c.y, h), __fadd_rn(c.z, h), 0.0f);
        }
    }
    ibox[2u * s] = lo;
    ibox[2u * s + 1u] = hi;
}

// Arrival counters of the climb: a node starts with its leaf children counted.
__global__ void k_icut_ibox_arrive(const Node* __restrict__ nodes, uint32_t m, uint32_t* __restrict__ arrive) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0 || j > m) return;
    arrive[j] = (nodes[j].c[0].cnt > 0 ? 1u : 0u) + (nodes[j].c[1].cnt > 0 ? 1u : 0u);
}

// Bottom-up climb (as the tree refit): from every node whose children are
// both leaves, the union of the children's influence boxes goes into the
// slot referencing the node unless interpolation stops at that slot (which
// keeps its own cube); the second arrival at a node continues upwards.
__global__ void k_icut_ibox_climb(const Node* __restrict__ nodes, uint32_t m, const uint32_t* __restrict__ pslot,
                                  uint32_t* arrive, float4* ibox) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    uint32_t j = 1u + t;
    if (!(nodes[j].c[0].cnt > 0 && nodes[j].c[1].cnt > 0)) return;
    for (int g = 0; g < kIcutMaxDepth; ++g) {
        const float4 a0 = __ldcg(ibox + 4u * j), a1 = __ldcg(ibox + 4u * j + 1u);
        const float4 b0 = __ldcg(ibox + 4u * j + 2u), b1 = __ldcg(ibox + 4u * j + 3u);
        const uint32_t s = pslot[j];
        const float4 own = __ldcg(ibox + 2u * s);
        if (own.w == 0.0f) {
            __stcg(ibox + 2u * s, make_float4(fminf(a0.x, b0.x), fminf(a0.y, b0.y), fminf(a0.z, b0.z), 0.0f));
            __stcg(ibox + 2u * s + 1u, make_float4(fmaxf(a1.x, b1.x), fmaxf(a1.y, b1.y), fmaxf(a1.z, b1.z), 0.0f));
        }
        if (s == 0u) break;
        const uint32_t p = s >> 1;
        __threadfence();
        if (atomicAdd(&arrive[p], 1u) != 1u) break;   // the sibling subtree is still climbing
        __threadfence();
        j = p;
    }
}

// Thread per query (Hilbert order when `order` is given): depth-first over the
// slots whose box lies within R of q, stopping at cut slots and leaves.
__global__ void __launch_bounds__(128) k_icut_interp(const Node* __restrict__ nodes, const float4* __restrict__ ibox,
                                                     const float4* __restrict__ center,
                                                     const float4* __restrict__ normal,
                                                     const float4* __restrict__ exact, const float4* __restrict__ qpos,
                                                     const float4* __restrict__ qnrm, const uint32_t* __restrict__ order,
                                                     uint32_t nq, float r2, float4* __restrict__ out, MapHeader* hdr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const uint32_t qo = order ? order[i] : i;
    const float4 q = qpos[qo];
    const float4 qn = qnrm[qo];
    if (!(isfinite(q.x) && isfinite(q.y) && isfinite(q.z))) {
        atomicOr(&hdr->errors, kErrQueryNonFinite);
        out[qo] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    double ax = 0.0, ay = 0.0, az = 0.0, ws = 0.0;
    uint32_t reached = 0;
    auto contribute = [&](uint32_t sid) {
        const float4 nn = __ldg(normal + sid);
        if (dot3_rn(nn.x, nn.y, nn.z, nn.x, nn.y, nn.z) == 0.0f) return;
        const float4 c = __ldg(center + sid);
        const float dist = __fsqrt_rn(d2_rn(q.x, q.y, q.z, c.x, c.y, c.z));
        if (!(c.w > 0.0f)) return;
        const float t = __fdiv_rn(dist, c.w);
        const float rbf = t <= 1.0f ? __fsub_rn(1.0f, __fmul_rn(t, t)) : 0.0f;
        const float w = __fmul_rn(rbf, fmaxf(0.0f, dot3_rn(nn.x, nn.y, nn.z, qn.x, qn.y, qn.z)));
        if (w == 0.0f) return;
        ++reached;
        const float4 e = __ldg(exact + sid);
        ax = __dadd_rn(ax, (double)w * (double)e.x);
        ay = __dadd_rn(ay, (double)w * (double)e.y);
        az = __dadd_rn(az, (double)w * (double)e.z);
        ws = __dadd_rn(ws, (double)w);
    };
    // a slot is entered when its box lies within R of q and its influence box holds q
    auto enter = [&](uint32_t sid, float4& ib_lo) -> bool {
        float lo[3], hi[3];
        uint32_t ref, cnt;
        slot_load(nodes, sid, lo, hi, ref, cnt);
        if (ref == kInvalid || !(box_lb(q.x, q.y, q.z, lo, hi) < r2)) return false;
        ib_lo = __ldg(ibox + 2u * sid);
        const float4 ib_hi = __ldg(ibox + 2u * sid + 1u);
        return q.x >= ib_lo.x && q.y >= ib_lo.y && q.z >= ib_lo.z && q.x <= ib_hi.x && q.y <= ib_hi.y &&
               q.z <= ib_hi.z;
    };
    uint32_t stack[kIcutStack];
    int sp = 0;
    float4 ib;
    if (enter(0u, ib)) {
        if (ib.w != 0.0f) contribute(0u);
        else stack[sp++] = 0u;
    }
    while (sp > 0) {
        const uint32_t j = slot_ref(nodes, stack[--sp]);   // internal: node j
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const uint32_t sid = 2u * j + (uint32_t)side;
            if (!enter(sid, ib)) continue;
            if (ib.w != 0.0f) {
                contribute(sid);
            } else if (sp < kIcutStack) {
                stack[sp++] = sid;
            } else {
                atomicOr(&hdr->errors, kErrStack);
            }
        }
    }
    float4 r = make_float4(0.f, 0.f, 0.f, (float)reached);
    if (ws != 0.0) {
        r.x = __double2float_rn(__ddiv_rn(ax, ws));
        r.y = __double2float_rn(__ddiv_rn(ay, ws));
        r.z = __double2float_rn(__ddiv_rn(az, ws));
    }
    out[qo] = r;
}

inline uint32_t blocks(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

int icut_prepare(const MapView& m, uint32_t num_nodes, const IcutBuffers& b, cudaStream_t st) {
    const uint32_t nslots = 2u * (num_nodes + 1u);
    // every walk up the tree ends at slot 0, also from a node no slot references
    cudaMemsetAsync(b.pslot, 0, ((size_t)num_nodes + 2) * sizeof(uint32_t), st);
    k_icut_parents<<<blocks(num_nodes + 1u, 256), 256, 0, st>>>(m.nodes, num_nodes, b.pslot);
    k_icut_slots<<<blocks(nslots, 256), 256, 0, st>>>(m.nodes, nslots, b.pslot, b.level, b.range, b.center, m.hdr);
    return 2;
}

int icut_normals(const MapView& m, uint32_t nslots, const float4* caller, const IcutBuffers& b, cudaStream_t st) {
    if (caller) {
        k_icut_copy_normals<<<blocks(nslots, 256), 256, 0, st>>>(caller, nslots, b.normal);
    } else {
        k_icut_normals<<<blocks(nslots * 32u, 256), 256, 0, st>>>(m.pow, nslots, b.range, b.normal);
    }
    return 1;
}

int icut_coarse(const MapView& m, uint32_t nslots, const IcutParams& p, const IcutBuffers& b, cudaStream_t st) {
    k_icut_estimate<<<blocks(nslots * 32u, 256), 256, 0, st>>>(m.pow, nslots, b.range, b.center, b.normal, b.est);
    if (p.use_leafs) {
        k_icut_leaves<<<blocks(nslots, 256), 256, 0, st>>>(m.nodes, nslots, b.coarse);
        return 2;
    }
    cudaMemsetAsync(b.acc, 0, 8 * sizeof(unsigned long long), st);
    k_icut_level_max<<<blocks(nslots, 256), 256, 0, st>>>(b.level, b.est, nslots, p.level_emin, b.acc);
    k_icut_level_sum<<<blocks(nslots, 256), 256, 0, st>>>(b.level, b.est, nslots, p.level_emin, b.acc);
    k_icut_mark0<<<blocks(nslots, 256), 256, 0, st>>>(b.level, b.est, nslots, b.acc, b.work[0]);
    k_icut_remove_parents<<<blocks(nslots, 256), 256, 0, st>>>(m.nodes, nslots, b.work[0], b.work[1]);
    k_icut_cover<<<blocks(nslots, 256), 256, 0, st>>>(m.nodes, nslots, b.pslot, b.work[1], b.coarse);
    return 6;
}

int icut_final(const MapView& m, uint32_t nslots, const IcutParams& p, const IcutBuffers& b, cudaStream_t st) {
    int nl = 0;
    cudaMemsetAsync(b.fin, 0, (size_t)nslots * sizeof(uint32_t), st);
    cudaMemcpyAsync(b.work[0], b.coarse, (size_t)nslots * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    int cur = 0;
    for (uint32_t it = 0; it < p.refine_iters; ++it) {
        cudaMemsetAsync(b.work[cur ^ 1], 0, (size_t)nslots * sizeof(uint32_t), st);
        k_icut_refine<<<blocks(nslots, 256), 256, 0, st>>>(m.nodes, nslots, b.est, b.exact, p.accuracy, b.work[cur],
                                                           b.work[cur ^ 1], b.fin);
        cur ^= 1;
        ++nl;
    }
    k_icut_finalize<<<blocks(nslots, 256), 256, 0, st>>>(nslots, b.work[cur], b.fin);
    // influence boxes of the final cut (b.work[cur ^ 1] is free: arrival counters)
    const uint32_t nodes_m = nslots / 2u - 1u;
    k_icut_ibox_own<<<blocks(nslots, 256), 256, 0, st>>>(m.nodes, nslots, b.pslot, b.fin, b.center, b.normal, b.ibox);
    if (nodes_m == 0) return nl + 2;
    k_icut_ibox_arrive<<<blocks(nodes_m + 1u, 256), 256, 0, st>>>(m.nodes, nodes_m, b.work[cur ^ 1]);
    k_icut_ibox_climb<<<blocks(nodes_m, 256), 256, 0, st>>>(m.nodes, nodes_m, b.pslot, b.work[cur ^ 1], b.ibox);
    return nl + 4;
}

int icut_interpolate(const MapView& m, const IcutBuffers& b, const float4* qpos, const float4* qnrm,
                     const uint32_t* order, uint32_t nq, float r2, float4* out, cudaStream_t st) {
    if (!nq) return 0;
    k_icut_interp<<<blocks(nq, 128), 128, 0, st>>>(m.nodes, b.ibox, b.center, b.normal, b.exact, qpos, qnrm, order, nq,
                                                   r2, out, m.hdr);
    return 1;
}

}  // namespace pm
