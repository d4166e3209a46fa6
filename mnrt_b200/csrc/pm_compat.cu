// pm_compat.cu -- the reference's own radius pipeline (PM_MODE_ZHOU_COMPAT).
//
// Restates KDTreePoint::PrecomputeQueryRadii / ComputeQueryRadii
// (KDTreePoint.cpp:187-248) and the kernels behind them
// (GPU/kdtree_point.cu:118-267, 295-546), then the range gather of
// dev_RangeSearch (GPU/photon_knn.cu:113-235):
//   1. node estimates: every tree slot (node) whose box radius (half
//      diagonal) is at most 0.5 R gets est = refine(centre, R); the others,
//      and all of them when the tree has fewer than 1000 slots, get +inf.
//      (The reference marks qualified nodes, unmarks their direct children
//      and re-marks two child levels, GPU/kdtree_point.cu:626-651; as child
//      boxes nest inside their parents, that is every qualified node.)
//   2. per query: est = min(R, min over the slots on the root-to-leaf path of
//      |q - centre| + est(slot)); the path follows the nearer child box (the
//      reference follows split planes; this tree has boxes);
//   3. refine(q, est): refine_iters rounds of a 32-bin histogram of the
//      distances d < r_max inside [r_min, r_max]; the first bin where the
//      cumulative count reaches k narrows [r_min, r_max] to that bin; counts
//      saturate at 0xfffe; the radius is the final r_max;
//   4. gather: every photon with d^2 < r^2 (strict), front test, filter;
//      r^2_used = max d^2 found when at least k were found, else r^2; fewer
//      than min_found photons -> 0.
// Arithmetic is FP32 with explicit roundings in a fixed order (the oracle
// restates the same steps on the exported tree); a histogram index that
// rounds to 32 (possible when d is just below r_max) goes to bin 31.
#include "pm_internal.h"

namespace pm {

namespace {

constexpr int kHist = 32;
constexpr int kCompatThreads = 64;
constexpr int kCompatStack = 128;

__device__ __forceinline__ void slot_of(const Node* nodes, uint32_t sid, float* lo, float* hi, uint32_t& ref,
                                        uint32_t& cnt) {
    const ChildSlot& s = nodes[sid >> 1].c[sid & 1u];
    lo[0] = s.lo[0]; lo[1] = s.lo[1]; lo[2] = s.lo[2];
    hi[0] = s.hi[0]; hi[1] = s.hi[1]; hi[2] = s.hi[2];
    ref = s.ref; cnt = s.cnt;
}

// Box centre and radius (half the diagonal), FP32 in a fixed order.
__device__ __forceinline__ void extent_of(const float* lo, const float* hi, float* c, float& rad) {
    float d2 = 0.0f;
    for (int a = 0; a < 3; ++a) {
        c[a] = __fmul_rn(__fadd_rn(lo[a], hi[a]), 0.5f);
        const float e = __fsub_rn(hi[a], lo[a]);
        d2 = a == 0 ? __fmul_rn(e, e) : __fadd_rn(d2, __fmul_rn(e, e));
    }
    rad = __fmul_rn(__fsqrt_rn(d2), 0.5f);
}

// Visits every photon with d^2 < r2 (DFS over the slots whose box lower
// bound is below r2).  f(tree position, d^2).  Returns false on stack overflow.
template <class F>
__device__ bool range_search(const Node* nodes, const float4* pos, float qx, float qy, float qz, float r2, F&& f) {
    uint32_t stack[kCompatStack];
    int sp = 0;
    stack[sp++] = 0u;   // slot 0 = the root slot of the super-root
    while (sp > 0) {
        const uint32_t sid = stack[--sp];
        float lo[3], hi[3];
        uint32_t ref, cnt;
        slot_of(nodes, sid, lo, hi, ref, cnt);
        if (ref == kInvalid) continue;
        if (!(box_lb(qx, qy, qz, lo, hi) < r2)) continue;
        if (cnt > 0) {
            for (uint32_t j = 0; j < cnt; ++j) {
                const float4 p = pos[ref + j];
                const float d2 = d2_rn(qx, qy, qz, p.x, p.y, p.z);
                if (d2 < r2) f(ref + j, d2);
            }
        } else {
            if (sp + 2 > kCompatStack) return false;
            stack[sp++] = (ref << 1) | 1u;
            stack[sp++] = ref << 1;
        }
    }
    return true;
}

// Zhou et al. 2008 histogram refinement of a query radius.
__device__ float refine_radius(const Node* nodes, const float4* pos, float qx, float qy, float qz, float radius_max,
                               uint32_t k, uint32_t iters, uint32_t* hist, bool& ok) {
    float r_min = 0.0f, r_max = radius_max;
    for (uint32_t it = 0; it < iters; ++it) {
        const float r = r_max;
        const float delta = __fsub_rn(r_max, r_min);
        if (!(delta > 0.0f)) break;
        for (int j = 0; j < kHist; ++j) hist[j * kCompatThreads] = 0;
        ok = range_search(nodes, pos, qx, qy, qz, __fmul_rn(r, r), [&](uint32_t, float d2) {
                 const float d = __fsqrt_rn(d2);
                 const float fi = __fdiv_rn(__fmul_rn(fmaxf(__fsub_rn(d, r_min), 0.0f), (float)kHist), delta);
                 uint32_t idx = (uint32_t)fi;
                 if (idx > kHist - 1) idx = kHist - 1;
                 uint32_t& h = hist[idx * kCompatThreads];
                 if (h < 0xfffeu) ++h;
             }) && ok;
        uint32_t m = kHist - 1, sum = 0;
        for (int j = 0; j < kHist; ++j) {
            sum += hist[j * kCompatThreads];
            if (sum >= k) { m = (uint32_t)j; break; }
        }
        const float inv = 1.0f / (float)kHist;
        const float old = r_min;
        r_min = __fadd_rn(old, __fmul_rn(__fmul_rn((float)m, delta), inv));
        r_max = __fadd_rn(old, __fmul_rn(__fmul_rn((float)(m + 1), delta), inv));
    }
    return r_max;
}

// One thread per slot; the slot count comes from the map header (2 per
// internal node plus the super-root's two), the launch covers an upper bound.
__global__ void __launch_bounds__(kCompatThreads) k_compat_nodes(const Node* nodes, const float4* pos, uint32_t max_slots,
                                                                 float rmax, uint32_t k, uint32_t iters, float* est,
                                                                 MapHeader* hdr) {
    __shared__ uint32_t s_hist[kHist * kCompatThreads];
    const uint32_t sid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t internal = hdr->num_nodes;
    const uint32_t nslots = 2 * (internal + 1);
    if (sid >= nslots || sid >= max_slots) return;
    const bool enabled = 2 * internal + 1 >= 1000;   // node estimates are skipped for small trees
    float e = INFINITY;
    float lo[3], hi[3];
    uint32_t ref, cnt;
    slot_of(nodes, sid, lo, hi, ref, cnt);
    if (enabled && ref != kInvalid) {
        float c[3], rad;
        extent_of(lo, hi, c, rad);
        if (rad <= __fmul_rn(0.5f, rmax)) {
            bool ok = true;
            e = refine_radius(nodes, pos, c[0], c[1], c[2], rmax, k, iters, s_hist + threadIdx.x, ok);
            if (!ok) atomicOr(&hdr->errors, kErrStack);
        }
    }
    est[sid] = e;
}

__device__ float query_radius(const Node* nodes, const float4* pos, const float* est, float qx, float qy, float qz,
                              float rmax, uint32_t k, uint32_t iters, uint32_t* hist, bool& ok) {
    float e = rmax;
    uint32_t sid = 0;
    for (int depth = 0; depth < 4096; ++depth) {
        float lo[3], hi[3];
        uint32_t ref, cnt;
        slot_of(nodes, sid, lo, hi, ref, cnt);
        if (ref == kInvalid) break;
        float c[3], rad;
        extent_of(lo, hi, c, rad);
        const float len = __fsqrt_rn(d2_rn(qx, qy, qz, c[0], c[1], c[2]));
        e = fminf(e, __fadd_rn(len, est[sid]));
        if (cnt > 0) break;
        float l0[3], h0[3], l1[3], h1[3];
        uint32_t r0, c0, r1, c1;
        slot_of(nodes, ref << 1, l0, h0, r0, c0);
        slot_of(nodes, (ref << 1) | 1u, l1, h1, r1, c1);
        const float b0 = r0 == kInvalid ? INFINITY : box_lb(qx, qy, qz, l0, h0);
        const float b1 = r1 == kInvalid ? INFINITY : box_lb(qx, qy, qz, l1, h1);
        sid = (ref << 1) | (b1 < b0 ? 1u : 0u);
    }
    return refine_radius(nodes, pos, qx, qy, qz, e, k, iters, hist, ok);
}

struct CompatArgs {
    const Node* nodes;
    const float4* pos;
    const float4* pow;
    const float* est;
    MapHeader* hdr;
    const float4* qpos;
    const float4* qnrm;
    uint32_t nq, k, iters, min_found;
    float rmax;
    int filter;
    float cone_k;
    float* out_radius;   // pm_compute_query_radii
    float4* out_rad;     // gather
    float* out_r2;
    uint32_t* out_count;
};

__global__ void __launch_bounds__(kCompatThreads) k_compat_query(CompatArgs a) {
    __shared__ uint32_t s_hist[kHist * kCompatThreads];
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.nq) return;
    const float4 qp = a.qpos[q];
    bool ok = true;
    float r = a.rmax;
    const bool finite = isfinite(qp.x) && isfinite(qp.y) && isfinite(qp.z);
    if (finite) r = query_radius(a.nodes, a.pos, a.est, qp.x, qp.y, qp.z, a.rmax, a.k, a.iters, s_hist + threadIdx.x, ok);
    else atomicOr(&a.hdr->errors, kErrQueryNonFinite);
    if (a.out_radius) a.out_radius[q] = r;
    if (a.out_rad) {
        const float4 qn = a.qnrm[q];
        const float r2 = __fmul_rn(r, r);
        uint32_t count = 0;
        float maxd2 = 0.0f;
        if (finite)
            ok = range_search(a.nodes, a.pos, qp.x, qp.y, qp.z, r2, [&](uint32_t, float d2) {
                     ++count;
                     maxd2 = fmaxf(maxd2, d2);
                 }) && ok;
        const float r2u = count >= a.k ? maxd2 : r2;
        float4 rad = make_float4(0.0f, 0.0f, 0.0f, (float)count);
        if (finite && count > 0 && count >= a.min_found && r2u > 0.0f) {
            const double r2d = (double)r2u;
            const double kc = (double)a.cone_k;
            // 2^40 / max flux: a range may hold far more than 128 photons
            const float scale = __fmul_rn(a.hdr->fix_scale, 1.220703125e-4f);
            long long c0 = 0, c1 = 0, c2 = 0;
            range_search(a.nodes, a.pos, qp.x, qp.y, qp.z, r2, [&](uint32_t t, float) {
                const float4 w = a.pow[t];
                if (!front_rn(qn.x, qn.y, qn.z, __float_as_uint(w.w))) return;
                const float4 p = a.pos[t];
                const double dx = (double)p.x - (double)qp.x, dy = (double)p.y - (double)qp.y,
                             dz = (double)p.z - (double)qp.z;
                const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                double wt = 1.0;
                if (a.filter == 1) wt = 1.0 - __dsqrt_rn(d2) / (kc * __dsqrt_rn(r2d));
                else if (a.filter == 2) wt = 1.0 - d2 / r2d;
                c0 += __double2ll_rn(wt * (double)w.x * (double)scale);
                c1 += __double2ll_rn(wt * (double)w.y * (double)scale);
                c2 += __double2ll_rn(wt * (double)w.z * (double)scale);
            });
            if (scale > 0.0f) {
                const double pi = 3.14159265358979323846;
                double norm = 1.0 / (pi * r2d);
                if (a.filter == 1) norm = 1.0 / ((1.0 - 2.0 / (3.0 * kc)) * pi * r2d);
                else if (a.filter == 2) norm = 2.0 / (pi * r2d);
                const double f = norm / (double)scale;
                rad.x = __double2float_rn((double)c0 * f);
                rad.y = __double2float_rn((double)c1 * f);
                rad.z = __double2float_rn((double)c2 * f);
            }
        }
        a.out_rad[q] = rad;
        if (a.out_r2) a.out_r2[q] = r2u;
        if (a.out_count) a.out_count[q] = count;
    }
    if (!ok) atomicOr(&a.hdr->errors, kErrStack);
}

}  // namespace

// est holds max_slots floats; max_slots >= 2 * (internal nodes + 1).
int compat_node_estimates(const MapView& m, uint32_t max_slots, float rmax, uint32_t k, uint32_t iters, float* est,
                          cudaStream_t st) {
    k_compat_nodes<<<(max_slots + kCompatThreads - 1) / kCompatThreads, kCompatThreads, 0, st>>>(
        m.nodes, m.pos, max_slots, rmax, k, iters, est, m.hdr);
    return 1;
}

int compat_query(const MapView& m, const float* est, const QueryParams& p, uint32_t iters, const float4* qpos,
                 const float4* qnrm, uint32_t nq, float* out_radius, const QueryOutputs& out, cudaStream_t st) {
    if (!nq) return 0;
    CompatArgs a;
    a.nodes = m.nodes; a.pos = m.pos; a.pow = m.pow; a.est = est; a.hdr = m.hdr;
    a.qpos = qpos; a.qnrm = qnrm; a.nq = nq; a.k = p.k; a.iters = iters; a.min_found = p.min_found;
    a.rmax = p.r; a.filter = p.filter; a.cone_k = p.cone_k;
    a.out_radius = out_radius; a.out_rad = out.rad; a.out_r2 = out.r2; a.out_count = out.count;
    k_compat_query<<<(nq + kCompatThreads - 1) / kCompatThreads, kCompatThreads, 0, st>>>(a);
    return 1;
}

}  // namespace pm
