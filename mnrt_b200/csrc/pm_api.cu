// pm_api.cu -- C ABI of the engine (include/pmgpu.h).
//
// A pm_map owns every device buffer it uses (photons in tree order, nodes,
// build and query scratch).  Arguments are validated before any CUDA call, so
// invalid calls fail the same way with or without a GPU.  Storage grows on
// demand outside stream capture; pm_reserve pre-sizes it for capture.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "pm_internal.h"
#include "pmgpu.h"

using namespace pm;

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct pm_map {
    // configuration
    uint32_t max_photons = 0;
    float scene_min[3] = {0, 0, 0}, scene_max[3] = {0, 0, 0};
    float r_max = 0.0f;
    // defaults: the fastest setting measured on the 1M-photon / 2M-query
    // workload (k = 100); pm_set_tuning / the autotuner override them
    uint32_t leaf_size = 32;
    int warps_per_block = 4;
    int rounds_per_chunk = 8;    // the smallest work chunk of the guided schedule, in rounds
    int queries_per_warp = 1;
    int kbuf_layout = PM_KBUF_WIDE;
    pm_alloc_fn alloc = nullptr;
    pm_free_fn free_fn = nullptr;
    void* alloc_user = nullptr;
    // state
    uint32_t n = 0;
    bool built = false;
    uint32_t cap_photons = 0;   // capacity of photon-sized buffers
    uint32_t cap_queries = 0;   // capacity of query-sized buffers
    // photon-sized
    DevBuf pos, pow, inv, nodes, hdr;
    DevBuf keys0, keys1, vals0, vals1, scratch, kfirst, klast, ksplit, kkeep, krank, parent, arrive, nleaf, partials;
    DevBuf wflag, wcnt, wfirst, wchild, wroot, wscan, rootmark;   // 32-wide tree
    // query-sized
    DevBuf qkeys0, qkeys1, qvals0, qvals1, qscratch, counter, fixq, qsorted;
    DevBuf stats;           // query counters (profiling level 2)
    // backward (pm_query_backward): pair sort, per-query records, segments,
    // FP64 running sums, and the forward outputs when the kNN is recomputed
    DevBuf bvals, bvals1, bkeys0, bkeys1, bscratch, blong, qrec, seg_start, seg_end, acc;
    DevBuf rnbr, rcnt, rr2, rrad;
    DevBuf gnrm, gest;        // pm_gather_for: flipped normals, estimates
    // PM_MODE_ZHOU_COMPAT: node radius estimates of the current tree, kept
    // for one (k, R, refinement rounds) until the next build
    DevBuf compat_est;
    // photons merged by pm_merge, built by pm_build_merged (PhotonData of the reference)
    DevBuf mpos, mpow, mflags, mrank, mscan;
    uint32_t merged_n = 0, cap_merged = 0;
    // illumination cut of the current tree (pm_icut_*): per-slot arrays
    DevBuf ic_pslot, ic_level, ic_range, ic_center, ic_normal, ic_est, ic_exact, ic_coarse, ic_fin, ic_work0, ic_work1,
        ic_acc, ic_ibox;
    uint32_t icut_slots = 0;
    // pm_build_query_host: device copies of host inputs, two copy streams, events
    DevBuf hs_pos, hs_pow, hs_qpos, hs_qnrm, hs_rad;
    cudaStream_t hs_in = nullptr, hs_out = nullptr;
    cudaEvent_t hs_ev[50] = {};   // photons in, done, and three per chunk
    uint64_t icut_prep_gen = ~0ull, icut_gen = ~0ull;
    uint64_t build_gen = 0, compat_gen = ~0ull;
    uint32_t compat_k = 0, compat_iters = 0;
    float compat_r = 0.0f;
    uint64_t cap_pairs = 0;
    uint32_t cap_bq = 0, cap_bn = 0, cap_rq = 0;
    uint32_t bwd_chunk = 0;   // max queries per backward chunk (0 = automatic)
    // profiling: events recorded on the call's stream when enabled
    bool profiling = false;
    int profile_level = 0;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // b0 b1 b2 q0 q1 q2
    bool have_build_ev = false, have_query_ev = false;
    uint32_t build_launches = 0, query_launches = 0;
    uint64_t launches = 0;
    char err[512] = {0};
};

namespace {

pm_status fail(pm_map* m, pm_status s, const char* fmt, ...) {
    if (m) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(m->err, sizeof(m->err), fmt, ap);
        va_end(ap);
    }
    return s;
}

pm_status check_cuda(pm_map* m, const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(m, PM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return PM_OK;
}

bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) { cudaGetLastError(); return false; }
    return cs != cudaStreamCaptureStatusNone;
}

void buf_free(pm_map* m, DevBuf& b) {
    if (b.ptr) {
        if (m->free_fn) m->free_fn(b.ptr, m->alloc_user);
        else cudaFree(b.ptr);
    }
    b.ptr = nullptr;
    b.bytes = 0;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

pm_status buf_ensure(pm_map* m, DevBuf& b, size_t bytes, const char* name) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return PM_OK;
    buf_free(m, b);
    void* p = nullptr;
    if (m->alloc) {
        if (m->alloc(&p, bytes, m->alloc_user) != 0 || !p)
            return fail(m, PM_ERR_OOM, "allocation of %zu bytes for %s failed (caller allocator)", bytes, name);
        if (!aligned16(p)) {   // float4 records and 64-bit scan words need it
            if (m->free_fn) m->free_fn(p, m->alloc_user);
            return fail(m, PM_ERR_INVALID, "the caller allocator returned a block for %s that is not 16-byte aligned",
                        name);
        }
    } else {
        const cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(m, e == cudaErrorMemoryAllocation ? PM_ERR_OOM : PM_ERR_CUDA,
                        "cudaMalloc of %zu bytes for %s failed: %s", bytes, name, cudaGetErrorString(e));
        }
    }
    b.ptr = p;
    b.bytes = bytes;
    return PM_OK;
}

template <class T> T* P(const DevBuf& b) { return reinterpret_cast<T*>(b.ptr); }


// Query counts stay below 2^31: slot, round and grid arithmetic in the
// kernels is 32-bit.
constexpr uint32_t kMaxQueries = 0x7fffffffu;

size_t sort_words(uint32_t n) { return sort_scratch_words(n) + 1 + scan_scratch_words(n) + 64; }

pm_status ensure_photon_capacity(pm_map* m, uint32_t n, cudaStream_t st) {
    if (n <= m->cap_photons && m->hdr.ptr) return PM_OK;
    if (capturing(st))
        return fail(m, PM_ERR_STATE, "map storage must grow to %u photons during stream capture; call pm_reserve first", n);
    const size_t cap = n ? n : 1;
    pm_status s;
#define ENSURE(buf, bytes) if ((s = buf_ensure(m, m->buf, (bytes), #buf)) != PM_OK) return s
    ENSURE(pos, cap * sizeof(float4));
    ENSURE(pow, cap * sizeof(float4));
    ENSURE(inv, cap * sizeof(uint32_t));
    ENSURE(nodes, (cap + 1) * sizeof(Node));
    ENSURE(hdr, sizeof(MapHeader));
    ENSURE(keys0, cap * sizeof(uint64_t));
    ENSURE(keys1, cap * sizeof(uint64_t));
    ENSURE(vals0, cap * sizeof(uint32_t));
    ENSURE(vals1, cap * sizeof(uint32_t));
    ENSURE(scratch, sort_words((uint32_t)cap) * sizeof(uint32_t));
    ENSURE(kfirst, cap * sizeof(uint32_t));
    ENSURE(klast, cap * sizeof(uint32_t));
    ENSURE(ksplit, cap * sizeof(uint32_t));
    ENSURE(kkeep, cap * sizeof(uint32_t));
    ENSURE(krank, cap * sizeof(uint32_t));
    ENSURE(parent, (cap + 1) * sizeof(uint32_t));
    ENSURE(arrive, (cap + 1) * sizeof(uint32_t));
    ENSURE(nleaf, (cap + 1) * sizeof(uint32_t));
    ENSURE(partials, (8 * 1184 + 16) * sizeof(uint32_t));
    ENSURE(wflag, cap * sizeof(uint32_t));
    ENSURE(wcnt, cap * sizeof(uint32_t));
    ENSURE(wfirst, cap * sizeof(uint32_t));
    ENSURE(wchild, (cap + 1) * 2 * sizeof(ChildSlot));
    ENSURE(wroot, sizeof(ChildSlot));
    ENSURE(wscan, wide_scan_words((uint32_t)cap) * sizeof(uint32_t));
    ENSURE(rootmark, (cap + 1) * sizeof(uint32_t));
#undef ENSURE
    m->cap_photons = (uint32_t)cap;
    return PM_OK;
}

pm_status ensure_query_capacity(pm_map* m, uint32_t nq, cudaStream_t st) {
    if (nq <= m->cap_queries && m->counter.ptr) return PM_OK;
    if (capturing(st))
        return fail(m, PM_ERR_STATE, "query storage must grow to %u queries during stream capture; call pm_reserve first", nq);
    const size_t cap = nq ? nq : 1;
    pm_status s;
#define ENSURE(buf, bytes) if ((s = buf_ensure(m, m->buf, (bytes), #buf)) != PM_OK) return s
    ENSURE(qkeys0, cap * sizeof(uint64_t));
    ENSURE(qkeys1, cap * sizeof(uint64_t));
    ENSURE(qvals0, cap * sizeof(uint32_t));
    ENSURE(qvals1, cap * sizeof(uint32_t));
    ENSURE(qscratch, sort_words((uint32_t)cap) * sizeof(uint32_t));
    ENSURE(counter, 64 * sizeof(uint32_t));
    ENSURE(fixq, cap * sizeof(uint32_t));
    ENSURE(qsorted, cap * 2 * sizeof(float4));   // query records in processing order (32 B per query)
#undef ENSURE
    m->cap_queries = (uint32_t)cap;
    return PM_OK;
}

pm_status validate_desc(pm_map* m, const pm_query_desc* d, bool exact_only, bool allow_icut = false) {
    if (!d) return fail(m, PM_ERR_INVALID, "query descriptor is NULL");
    if (d->k == 0) return fail(m, PM_ERR_INVALID, "k must be >= 1");
    if (d->k > PM_MAX_K) return fail(m, PM_ERR_UNSUPPORTED, "k = %u exceeds PM_MAX_K = %u", d->k, PM_MAX_K);
    if (!(d->r_max > 0.0f) || !std::isfinite(d->r_max))
        return fail(m, PM_ERR_INVALID, "r_max must be finite and > 0 (got %g)", (double)d->r_max);
    if (d->filter < PM_FILTER_BOX || d->filter > PM_FILTER_EPANECHNIKOV)
        return fail(m, PM_ERR_INVALID, "unknown filter %d", d->filter);
    if (d->filter == PM_FILTER_CONE && !(d->cone_k >= 1.0f && std::isfinite(d->cone_k)))
        return fail(m, PM_ERR_INVALID, "cone_k must be finite and >= 1 (got %g)", (double)d->cone_k);
    if (d->mode == PM_MODE_ICUT && !allow_icut)
        return fail(m, PM_ERR_INVALID, "PM_MODE_ICUT is a pm_gather_for mode only");
    if (d->mode != PM_MODE_EXACT && d->mode != PM_MODE_ZHOU_COMPAT && d->mode != PM_MODE_ICUT)
        return fail(m, PM_ERR_INVALID, "unknown mode %d", d->mode);
    if (exact_only && d->mode == PM_MODE_ZHOU_COMPAT)
        return fail(m, PM_ERR_INVALID, "this entry point supports PM_MODE_EXACT only");
    if (d->order != PM_ORDER_SORTED && d->order != PM_ORDER_AS_GIVEN)
        return fail(m, PM_ERR_INVALID, "unknown query order %d", d->order);
    return PM_OK;
}

MapView view_of(pm_map* m) {
    MapView v;
    v.pos = P<float4>(m->pos);
    v.pow = P<float4>(m->pow);
    v.inv = P<uint32_t>(m->inv);
    v.wchild = P<ChildSlot>(m->wchild);
    v.wroot = P<ChildSlot>(m->wroot);
    v.nodes = P<Node>(m->nodes);
    v.hdr = P<MapHeader>(m->hdr);
    v.n = m->n;
    return v;
}

WideBuffers wide_of(pm_map* m) {
    WideBuffers w;
    w.wflag = P<uint32_t>(m->wflag); w.wcnt = P<uint32_t>(m->wcnt);
    w.wfirst = P<uint32_t>(m->wfirst); w.wchild = P<ChildSlot>(m->wchild); w.wroot = P<ChildSlot>(m->wroot);
    w.scratch = P<uint32_t>(m->wscan);
    return w;
}

QueryTuning tuning_of(const pm_map* m) {
    QueryTuning t;
    t.layout = m->kbuf_layout;
    t.queries_per_warp = m->queries_per_warp;
    t.warps_per_block = m->warps_per_block;
    t.rounds_per_chunk = m->rounds_per_chunk;
    t.stats = (m->profile_level >= 2 && m->stats.ptr) ? P<unsigned long long>(m->stats) : nullptr;
    return t;
}

QueryParams params_of(const pm_query_desc* d) {
    QueryParams p;
    p.k = d->k;
    p.r = d->r_max;
    p.r2 = d->r_max * d->r_max;
    p.filter = d->filter;
    p.cone_k = d->filter == PM_FILTER_CONE ? d->cone_k : 1.0f;
    p.min_found = d->min_found;
    return p;
}

// Hilbert order of the queries (returns the permutation or nullptr).
const uint32_t* sort_queries(pm_map* m, const float4* qpos, uint32_t nq, cudaStream_t st, int* launches,
                             bool hilbert = true) {
    *launches += query_order_keys(qpos, nq, P<MapHeader>(m->hdr), P<uint32_t>(m->qkeys0), P<uint32_t>(m->qvals0), st,
                                  hilbert);
    uint32_t* keys[2] = {P<uint32_t>(m->qkeys0), P<uint32_t>(m->qkeys1)};
    uint32_t* vals[2] = {P<uint32_t>(m->qvals0), P<uint32_t>(m->qvals1)};
    const int cur = radix_sort_pairs32(keys, vals, nq, kQueryKeyBits, P<uint32_t>(m->qscratch), st, launches);
    return vals[cur];
}

}  // namespace

extern "C" {

int pm_abi_version(void) { return 1; }

const char* pm_status_string(pm_status s) {
    switch (s) {
        case PM_OK: return "ok";
        case PM_ERR_INVALID: return "invalid argument";
        case PM_ERR_CUDA: return "CUDA error";
        case PM_ERR_OOM: return "out of device memory";
        case PM_ERR_STATE: return "invalid state";
        case PM_ERR_DEVICE: return "device-side error";
        case PM_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* pm_last_error(const pm_map* m) { return m ? m->err : "null handle"; }

pm_status pm_create(pm_map** out, uint32_t max_photons, const float* aabb_min, const float* aabb_max, float r_max) {
    if (!out) return PM_ERR_INVALID;
    *out = nullptr;
    if (!(r_max > 0.0f) || !std::isfinite(r_max)) return PM_ERR_INVALID;
    pm_map* m = new (std::nothrow) pm_map();
    if (!m) return PM_ERR_OOM;
    m->max_photons = max_photons;
    for (int a = 0; a < 3; ++a) {
        m->scene_min[a] = aabb_min ? aabb_min[a] : 0.0f;
        m->scene_max[a] = aabb_max ? aabb_max[a] : 0.0f;
    }
    m->r_max = r_max;
    *out = m;
    return PM_OK;
}

pm_status pm_destroy(pm_map* m) {
    if (!m) return PM_ERR_INVALID;
    DevBuf* all[] = {&m->pos, &m->pow, &m->inv, &m->nodes, &m->hdr, &m->keys0, &m->keys1, &m->vals0, &m->vals1,
                     &m->scratch, &m->kfirst, &m->klast, &m->ksplit, &m->kkeep, &m->krank, &m->parent,
                     &m->arrive, &m->nleaf, &m->partials, &m->wflag, &m->wcnt, &m->wfirst,
                     &m->wchild, &m->wroot, &m->wscan, &m->rootmark, &m->qkeys0, &m->qkeys1, &m->qvals0, &m->qvals1,
                     &m->qscratch, &m->counter, &m->fixq, &m->qsorted, &m->stats, &m->bvals, &m->bvals1, &m->bkeys0, &m->bkeys1, &m->blong,
                     &m->bscratch, &m->qrec, &m->seg_start, &m->seg_end, &m->acc, &m->rnbr,
                     &m->rcnt, &m->rr2, &m->rrad, &m->gnrm, &m->gest, &m->compat_est, &m->mpos, &m->mpow, &m->mflags,
                     &m->mrank, &m->mscan, &m->ic_pslot, &m->ic_level, &m->ic_range, &m->ic_center,
                     &m->ic_normal, &m->ic_est, &m->ic_exact, &m->ic_coarse, &m->ic_fin, &m->ic_work0, &m->ic_work1,
                     &m->ic_acc, &m->ic_ibox, &m->hs_pos, &m->hs_pow, &m->hs_qpos, &m->hs_qnrm, &m->hs_rad};
    for (DevBuf* b : all) buf_free(m, *b);
    for (cudaEvent_t& e : m->hs_ev)
        if (e) cudaEventDestroy(e);
    if (m->hs_in) cudaStreamDestroy(m->hs_in);
    if (m->hs_out) cudaStreamDestroy(m->hs_out);
    for (cudaEvent_t& e : m->ev)
        if (e) cudaEventDestroy(e);
    delete m;
    return PM_OK;
}

pm_status pm_set_allocator(pm_map* m, pm_alloc_fn alloc, pm_free_fn free_fn, void* user) {
    if (!m) return PM_ERR_INVALID;
    if ((alloc == nullptr) != (free_fn == nullptr))
        return fail(m, PM_ERR_INVALID, "alloc and free must both be set or both be NULL");
    if (m->hdr.ptr || m->counter.ptr) return fail(m, PM_ERR_STATE, "allocator must be set before the first build or query");
    m->alloc = alloc;
    m->free_fn = free_fn;
    m->alloc_user = user;
    return PM_OK;
}

pm_status pm_set_tuning(pm_map* m, uint32_t leaf_size, int warps_per_block, int rounds_per_chunk,
                        int queries_per_warp, int kbuf_layout) {
    if (!m) return PM_ERR_INVALID;
    if (leaf_size < 1 || leaf_size > kLeafMax) return fail(m, PM_ERR_INVALID, "leaf_size must be in [1, %u]", kLeafMax);
    if (warps_per_block < 1 || warps_per_block > 8) return fail(m, PM_ERR_INVALID, "warps_per_block must be in [1, 8]");
    if (rounds_per_chunk < 1 || rounds_per_chunk > 4096) return fail(m, PM_ERR_INVALID, "rounds_per_chunk must be in [1, 4096]");
    if (queries_per_warp != 1 && queries_per_warp != 2 && queries_per_warp != 4 && queries_per_warp != 8)
        return fail(m, PM_ERR_INVALID, "queries_per_warp must be 1, 2, 4 or 8");
    if (kbuf_layout != PM_KBUF_HEAP && kbuf_layout != PM_KBUF_GROUP && kbuf_layout != PM_KBUF_WIDE)
        return fail(m, PM_ERR_INVALID, "unknown k-buffer layout %d", kbuf_layout);
    m->leaf_size = leaf_size;
    m->warps_per_block = warps_per_block;
    m->rounds_per_chunk = rounds_per_chunk;
    m->queries_per_warp = queries_per_warp;
    m->kbuf_layout = kbuf_layout;
    return PM_OK;
}

pm_status pm_reserve(pm_map* m, uint32_t max_photons, uint32_t max_queries) {
    if (!m) return PM_ERR_INVALID;
    pm_status s = ensure_photon_capacity(m, max_photons, nullptr);
    if (s != PM_OK) return s;
    return ensure_query_capacity(m, max_queries, nullptr);
}

pm_status pm_build(pm_map* m, const float* d_pos4, const float* d_pow4, uint32_t n, int format, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (format != PM_PHOTONS_REFERENCE && format != PM_PHOTONS_PACKED)
        return fail(m, PM_ERR_INVALID, "unknown photon format %d", format);
    if (n > 0 && (!d_pos4 || !d_pow4)) return fail(m, PM_ERR_INVALID, "photon arrays must be non-NULL when n > 0");
    if (n > 0 && (!aligned16(d_pos4) || !aligned16(d_pow4)))
        return fail(m, PM_ERR_INVALID, "photon arrays must be 16-byte aligned");
    if (m->max_photons && n > m->max_photons)
        return fail(m, PM_ERR_INVALID, "n = %u exceeds the map's max_photons = %u", n, m->max_photons);
    if (n > 0x7fffffffu) return fail(m, PM_ERR_UNSUPPORTED, "n = %u exceeds 2^31 - 1 photons", n);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    pm_status s = ensure_photon_capacity(m, n, st);
    if (s != PM_OK) return s;
    BuildBuffers bb;
    bb.keys[0] = P<uint64_t>(m->keys0); bb.keys[1] = P<uint64_t>(m->keys1);
    bb.vals[0] = P<uint32_t>(m->vals0); bb.vals[1] = P<uint32_t>(m->vals1);
    bb.scratch = P<uint32_t>(m->scratch);
    bb.kfirst = P<uint32_t>(m->kfirst); bb.klast = P<uint32_t>(m->klast); bb.ksplit = P<uint32_t>(m->ksplit);
    bb.kkeep = P<uint32_t>(m->kkeep); bb.krank = P<uint32_t>(m->krank);
    bb.parent = P<uint32_t>(m->parent); bb.arrive = P<uint32_t>(m->arrive); bb.nleaf = P<uint32_t>(m->nleaf);
    bb.partials = P<uint32_t>(m->partials); bb.num_partials = 1184;
    const bool prof = m->profiling && !capturing(st);
    if (prof) cudaEventRecord(m->ev[0], st);
    const int nl = build_map(reinterpret_cast<const float4*>(d_pos4), reinterpret_cast<const float4*>(d_pow4), n,
                             format, m->leaf_size, P<float4>(m->pos), P<float4>(m->pow), P<uint32_t>(m->inv), P<Node>(m->nodes),
                             P<MapHeader>(m->hdr), bb, wide_of(m), st, prof ? m->ev[1] : nullptr);
    if (prof) cudaEventRecord(m->ev[2], st);
    m->have_build_ev = prof;
    m->build_launches = (uint32_t)nl;
    m->launches += (uint64_t)nl;
    s = check_cuda(m, "pm_build");
    if (s != PM_OK) return s;
    m->n = n;
    m->built = true;
    ++m->build_gen;
    return PM_OK;
}

static pm_status query_common(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4,
                              uint32_t nq, float* d_rad4, bool exact_only) {
    if (!m) return PM_ERR_INVALID;
    pm_status s = validate_desc(m, desc, exact_only);
    if (s != PM_OK) return s;
    if (nq > kMaxQueries) return fail(m, PM_ERR_UNSUPPORTED, "nq = %u exceeds 2^31 - 1 queries", nq);
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    if (nq > 0 && (!d_qpos4 || !d_qnrm4 || !d_rad4))
        return fail(m, PM_ERR_INVALID, "query positions, normals and radiance output must be non-NULL");
    if (nq > 0 && (!aligned16(d_qpos4) || !aligned16(d_qnrm4) || !aligned16(d_rad4)))
        return fail(m, PM_ERR_INVALID, "query and radiance arrays must be 16-byte aligned");
    return PM_OK;
}

static pm_status compat_run(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4,
                            uint32_t nq, float* d_radius, float* d_rad4, float* d_r2, uint32_t* d_count, cudaStream_t st) {
    if (nq == 0) return PM_OK;
    const uint32_t iters = desc->refine_iters;
    if (iters > 64) return fail(m, PM_ERR_INVALID, "refine_iters must be at most 64");
    const uint32_t max_slots = 2 * (m->cap_photons + 1);
    if (m->compat_gen != m->build_gen || m->compat_k != desc->k || m->compat_r != desc->r_max ||
        m->compat_iters != iters) {
        if (m->compat_est.bytes < (size_t)max_slots * sizeof(float)) {
            if (capturing(st)) return fail(m, PM_ERR_STATE, "compat storage must grow during stream capture");
            pm_status s = buf_ensure(m, m->compat_est, (size_t)max_slots * sizeof(float), "compat node estimates");
            if (s != PM_OK) return s;
        }
        m->launches += (uint64_t)compat_node_estimates(view_of(m), max_slots, desc->r_max, desc->k, iters,
                                                       P<float>(m->compat_est), st);
        m->compat_gen = m->build_gen; m->compat_k = desc->k; m->compat_r = desc->r_max; m->compat_iters = iters;
    }
    QueryOutputs out{reinterpret_cast<float4*>(d_rad4), nullptr, d_r2, d_count};
    m->launches += (uint64_t)compat_query(view_of(m), P<float>(m->compat_est), params_of(desc), iters,
                                          reinterpret_cast<const float4*>(d_qpos4),
                                          reinterpret_cast<const float4*>(d_qnrm4), nq, d_radius, out, st);
    return check_cuda(m, "PM_MODE_ZHOU_COMPAT");
}

// The exact query of validated arguments: Hilbert sort of the positions,
// then the search.  nrm_ready (optional) is an event the search waits for
// after the sort, so a caller still copying the normals in overlaps the sort
// with that copy.
static pm_status query_exact_run(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4,
                                 uint32_t nq, float* d_rad4, uint32_t* d_nbr, float* d_r2, uint32_t* d_count,
                                 cudaStream_t st, cudaEvent_t nrm_ready) {
    if (nq == 0) return PM_OK;
    pm_status s = ensure_query_capacity(m, nq, st);
    if (s != PM_OK) return s;
    const float4* qpos = reinterpret_cast<const float4*>(d_qpos4);
    const bool prof = m->profiling && !capturing(st);
    if (prof) cudaEventRecord(m->ev[3], st);
    int nl = 0;
    const uint32_t* order = desc->order == PM_ORDER_SORTED ? sort_queries(m, qpos, nq, st, &nl) : nullptr;
    if (prof) cudaEventRecord(m->ev[4], st);
    if (nrm_ready) cudaStreamWaitEvent(st, nrm_ready, 0);
    QueryOutputs out{reinterpret_cast<float4*>(d_rad4), d_nbr, d_r2, d_count};
    QueryTuning t = tuning_of(m);
    if (order && t.layout == 2) {
        // the 32-byte query records in processing order, so the search reads them
        // sequentially instead of through the permutation (after the normals have
        // arrived: the sort above only needs the positions); 6.97 -> 6.90 ms for
        // the plain workload's search, this launch included
        nl += gather_queries(order, qpos, reinterpret_cast<const float4*>(d_qnrm4), nq, P<float4>(m->qsorted), st);
        t.qsorted = P<float4>(m->qsorted);
    }
    nl += query_knn(view_of(m), params_of(desc), qpos, reinterpret_cast<const float4*>(d_qnrm4), order, nq, out,
                    P<uint32_t>(m->counter), P<uint32_t>(m->fixq), t, st);
    if (prof) cudaEventRecord(m->ev[5], st);
    m->have_query_ev = prof;
    m->query_launches = (uint32_t)nl;
    m->launches += (uint64_t)nl;
    return check_cuda(m, "pm_query");
}

pm_status pm_query(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4, uint32_t nq,
                   float* d_rad4, uint32_t* d_nbr, float* d_r2, uint32_t* d_count, void* stream) {
    pm_status s = query_common(m, desc, d_qpos4, d_qnrm4, nq, d_rad4, false);
    if (s != PM_OK) return s;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (desc->mode == PM_MODE_ZHOU_COMPAT) {
        if (d_nbr) return fail(m, PM_ERR_INVALID, "PM_MODE_ZHOU_COMPAT returns no neighbour lists (d_nbr must be NULL)");
        return compat_run(m, desc, d_qpos4, d_qnrm4, nq, nullptr, d_rad4, d_r2, d_count, st);
    }
    return query_exact_run(m, desc, d_qpos4, d_qnrm4, nq, d_rad4, d_nbr, d_r2, d_count, st, nullptr);
}

// Device address of a page-locked host array (cudaHostAlloc /
// cudaHostRegister, mapped under unified addressing), or nullptr.
static void* host_mapped(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

pm_status pm_build_query_host(pm_map* m, const float* h_pos4, const float* h_pow4, uint32_t n, int format,
                              const pm_query_desc* desc, const float* h_qpos4, const float* h_qnrm4, uint32_t nq,
                              float* h_rad4, uint32_t chunks, void* stream) {
    if (!m) return PM_ERR_INVALID;
    pm_status s = validate_desc(m, desc, true);
    if (s != PM_OK) return s;
    if (format != PM_PHOTONS_REFERENCE && format != PM_PHOTONS_PACKED)
        return fail(m, PM_ERR_INVALID, "unknown photon format %d", format);
    if (chunks == 0) chunks = 1;
    if (chunks > 16) return fail(m, PM_ERR_INVALID, "chunks must be at most 16");
    if (n > 0 && (!h_pos4 || !h_pow4)) return fail(m, PM_ERR_INVALID, "photon arrays must be non-NULL when n > 0");
    if (nq > kMaxQueries) return fail(m, PM_ERR_UNSUPPORTED, "nq = %u exceeds 2^31 - 1 queries", nq);
    if (nq > 0 && (!h_qpos4 || !h_qnrm4 || !h_rad4))
        return fail(m, PM_ERR_INVALID, "query positions, normals and radiance output must be non-NULL");
    if (m->max_photons && n > m->max_photons)
        return fail(m, PM_ERR_INVALID, "n = %u exceeds the map's max_photons = %u", n, m->max_photons);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (capturing(st)) return fail(m, PM_ERR_STATE, "pm_build_query_host cannot run during stream capture");
    if (!m->hs_in) {
        if (cudaStreamCreateWithFlags(&m->hs_in, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&m->hs_out, cudaStreamNonBlocking) != cudaSuccess)
            return check_cuda(m, "pm_build_query_host: streams");
        for (cudaEvent_t& e : m->hs_ev)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                return check_cuda(m, "pm_build_query_host: events");
    }
    const size_t pb = (size_t)(n ? n : 1) * sizeof(float4), qb = (size_t)(nq ? nq : 1) * sizeof(float4);
    if ((s = buf_ensure(m, m->hs_pos, pb, "hs_pos")) != PM_OK || (s = buf_ensure(m, m->hs_pow, pb, "hs_pow")) != PM_OK ||
        (s = buf_ensure(m, m->hs_qpos, qb, "hs_qpos")) != PM_OK ||
        (s = buf_ensure(m, m->hs_qnrm, qb, "hs_qnrm")) != PM_OK || (s = buf_ensure(m, m->hs_rad, qb, "hs_rad")) != PM_OK)
        return s;
    float4* dpos = P<float4>(m->hs_pos);
    float4* dpow = P<float4>(m->hs_pow);
    float4* dqp = P<float4>(m->hs_qpos);
    float4* dqn = P<float4>(m->hs_qnrm);
    float4* drad = P<float4>(m->hs_rad);
    // A page-locked, 16-byte aligned radiance array is written in place by the query kernel
    // (each estimate once, 16 bytes over PCIe while the search runs), which
    // takes the download off the critical path: 9.83 -> 9.27 ms end to end on
    // the plain workload.  A pageable one goes through a device copy.  The
    // normals are always copied in: read in place as well, they queue behind
    // the posted radiance writes on the link (12.76 ms with both in place;
    // 9.57 ms with the normals alone).
    void* const rad_mapped = (nq > 0 && aligned16(h_rad4)) ? host_mapped(h_rad4) : nullptr;
    const bool rad_in_place = rad_mapped != nullptr;
    if (rad_in_place) drad = reinterpret_cast<float4*>(rad_mapped);
    cudaEvent_t ev_photons = m->hs_ev[0], ev_done = m->hs_ev[1];
    // photons in, then the queries in pieces behind them on the copy stream
    if (n) {
        cudaMemcpyAsync(dpos, h_pos4, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dpow, h_pow4, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, st);
    }
    cudaEventRecord(ev_photons, st);
    cudaStreamWaitEvent(m->hs_in, ev_photons, 0);
    if (nq < chunks) chunks = nq ? nq : 1;
    uint32_t bounds[17];
    for (uint32_t c = 0; c <= chunks; ++c) bounds[c] = (uint32_t)(((uint64_t)nq * c) / chunks);
    for (uint32_t c = 0; c < chunks; ++c) {   // positions first: the piece's sort needs only them
        const size_t off = bounds[c], len = bounds[c + 1] - bounds[c];
        if (len)
            cudaMemcpyAsync(dqp + off, reinterpret_cast<const float4*>(h_qpos4) + off, len * sizeof(float4),
                            cudaMemcpyHostToDevice, m->hs_in);
        cudaEventRecord(m->hs_ev[2 + 3 * c], m->hs_in);
        if (len)
            cudaMemcpyAsync(dqn + off, reinterpret_cast<const float4*>(h_qnrm4) + off, len * sizeof(float4),
                            cudaMemcpyHostToDevice, m->hs_in);
        cudaEventRecord(m->hs_ev[3 + 3 * c], m->hs_in);
    }
    s = check_cuda(m, "pm_build_query_host: copies in");
    if (s != PM_OK) return s;
    s = pm_build(m, reinterpret_cast<const float*>(dpos), reinterpret_cast<const float*>(dpow), n, format, stream);
    if (s != PM_OK) return s;
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    // each piece is sorted once its positions have arrived and searched once
    // its normals have; its radiance leaves on the second stream
    for (uint32_t c = 0; c < chunks; ++c) {
        const size_t off = bounds[c], len = bounds[c + 1] - bounds[c];
        cudaStreamWaitEvent(st, m->hs_ev[2 + 3 * c], 0);
        if (len) {
            s = query_exact_run(m, desc, reinterpret_cast<const float*>(dqp + off),
                                reinterpret_cast<const float*>(dqn + off), (uint32_t)len,
                                reinterpret_cast<float*>(drad + off), nullptr, nullptr, nullptr, st, m->hs_ev[3 + 3 * c]);
            if (s != PM_OK) return s;
        } else {
            cudaStreamWaitEvent(st, m->hs_ev[3 + 3 * c], 0);
        }
        cudaEventRecord(m->hs_ev[4 + 3 * c], st);
        cudaStreamWaitEvent(m->hs_out, m->hs_ev[4 + 3 * c], 0);
        if (len && !rad_in_place)
            cudaMemcpyAsync(reinterpret_cast<float4*>(h_rad4) + off, drad + off, len * sizeof(float4),
                            cudaMemcpyDeviceToHost, m->hs_out);
    }
    cudaEventRecord(ev_done, m->hs_out);
    cudaStreamWaitEvent(st, ev_done, 0);
    return check_cuda(m, "pm_build_query_host");
}

pm_status pm_query_bruteforce(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4,
                              uint32_t nq, float* d_rad4, uint32_t* d_nbr, float* d_r2, uint32_t* d_count,
                              void* stream) {
    pm_status s = query_common(m, desc, d_qpos4, d_qnrm4, nq, d_rad4, true);
    if (s != PM_OK) return s;
    if (nq == 0) return PM_OK;
    QueryOutputs out{reinterpret_cast<float4*>(d_rad4), d_nbr, d_r2, d_count};
    m->launches += (uint64_t)query_bruteforce(view_of(m), params_of(desc), reinterpret_cast<const float4*>(d_qpos4),
                                              reinterpret_cast<const float4*>(d_qnrm4), nq, out,
                                              reinterpret_cast<cudaStream_t>(stream));
    return check_cuda(m, "pm_query_bruteforce");
}

pm_status pm_set_backward_chunk(pm_map* m, uint32_t max_queries) {
    if (!m) return PM_ERR_INVALID;
    m->bwd_chunk = max_queries;
    return PM_OK;
}

static pm_status ensure_bwd_capacity(pm_map* m, uint32_t chunk_q, uint32_t k, bool recompute, bool chunked,
                                     cudaStream_t st) {
    const uint64_t pairs = (uint64_t)chunk_q * k;
    const uint32_t n = m->n ? m->n : 1;
    const uint64_t pc = pairs ? pairs : 1;
    // the sort path's buffers when the largest chunk takes it
    const bool sort_path = bwd_sort_path(pairs, n);
    const size_t scratch_bytes = bwd_scratch_words(n, pc, sort_path) * sizeof(uint32_t);
    const bool grow = pairs > m->cap_pairs || chunk_q > m->cap_bq || n > m->cap_bn || (chunked && !m->acc.ptr) ||
                      (chunked && m->acc.bytes < (size_t)n * 6 * sizeof(double)) ||
                      m->bscratch.bytes < scratch_bytes || (sort_path && m->bkeys1.bytes < pc * sizeof(uint32_t)) ||
                      (recompute && (chunk_q > m->cap_rq || !m->rnbr.ptr || m->rnbr.bytes < pairs * 4));
    if (!grow) return PM_OK;
    if (capturing(st))
        return fail(m, PM_ERR_STATE, "backward storage must grow during stream capture; run one backward first");
    pm_status s;
#define ENSURE(buf, bytes) if ((s = buf_ensure(m, m->buf, (bytes), #buf)) != PM_OK) return s
    const size_t qc = chunk_q ? chunk_q : 1;
    ENSURE(bvals, pc * sizeof(uint32_t));
    if (sort_path) {
        ENSURE(bvals1, pc * sizeof(uint32_t));
        ENSURE(bkeys0, pc * sizeof(uint32_t));
        ENSURE(bkeys1, pc * sizeof(uint32_t));
    }
    ENSURE(bscratch, scratch_bytes);
    ENSURE(blong, ((size_t)n + 1) * sizeof(uint32_t));
    ENSURE(qrec, qc * sizeof(BwdQuery));
    ENSURE(seg_start, (size_t)n * sizeof(uint32_t));
    ENSURE(seg_end, (size_t)n * sizeof(uint32_t));
    if (chunked) ENSURE(acc, (size_t)n * 6 * sizeof(double));
    if (recompute) {
        ENSURE(rnbr, pc * sizeof(uint32_t));
        ENSURE(rcnt, qc * sizeof(uint32_t));
        ENSURE(rr2, qc * sizeof(float));
        ENSURE(rrad, qc * sizeof(float4));
        if (chunk_q > m->cap_rq) m->cap_rq = chunk_q;
    }
#undef ENSURE
    if (pairs > m->cap_pairs) m->cap_pairs = pairs;
    if (chunk_q > m->cap_bq) m->cap_bq = chunk_q;
    if (n > m->cap_bn) m->cap_bn = n;
    return PM_OK;
}

pm_status pm_query_backward(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4,
                            uint32_t nq, const float* d_grad_rad4, const uint32_t* d_nbr, const float* d_r2,
                            const uint32_t* d_count, float* d_grad_pow4, float* d_grad_pos4, void* stream) {
    (void)d_r2;   // r^2 is re-derived in FP64 from the k-th neighbour
    if (!m) return PM_ERR_INVALID;
    pm_status s = validate_desc(m, desc, true);
    if (s != PM_OK) return s;
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    if (!d_grad_pow4 && !d_grad_pos4) return fail(m, PM_ERR_INVALID, "both gradient outputs are NULL");
    if ((d_grad_pow4 && !aligned16(d_grad_pow4)) || (d_grad_pos4 && !aligned16(d_grad_pos4)))
        return fail(m, PM_ERR_INVALID, "gradient arrays must be 16-byte aligned");
    if (nq > kMaxQueries) return fail(m, PM_ERR_UNSUPPORTED, "nq = %u exceeds 2^31 - 1 queries", nq);
    if (nq > 0 && (!d_qpos4 || !d_qnrm4 || !d_grad_rad4))
        return fail(m, PM_ERR_INVALID, "query positions, normals and dL/dE must be non-NULL");
    if (nq > 0 && (!aligned16(d_qpos4) || !aligned16(d_qnrm4) || !aligned16(d_grad_rad4)))
        return fail(m, PM_ERR_INVALID, "query and dL/dE arrays must be 16-byte aligned");
    if (m->n == 0) return PM_OK;   // no photons: nothing to differentiate
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t k = desc->k;
    const uint64_t kMaxPairs = 1ull << 27;   // neighbour pairs per chunk (512 MB of pair slots; 2 GB on the sort path)
    uint32_t chunk = (uint32_t)(kMaxPairs / k);
    if (m->bwd_chunk) chunk = m->bwd_chunk < chunk ? m->bwd_chunk : chunk;
    if (nq > 0 && chunk > nq) chunk = nq;
    if (chunk == 0) chunk = 1;
    const uint32_t nchunks = nq ? (nq + chunk - 1) / chunk : 1;
    const bool recompute = d_nbr == nullptr;
    s = ensure_bwd_capacity(m, chunk, k, recompute, nchunks > 1, st);
    if (s != PM_OK) return s;
    const bool sorted = desc->order == PM_ORDER_SORTED;
    if (recompute || sorted) {
        s = ensure_query_capacity(m, chunk, st);
        if (s != PM_OK) return s;
    }
    BwdArgs a;
    a.pos = P<float4>(m->pos); a.pow = P<float4>(m->pow); a.inv = P<uint32_t>(m->inv);
    a.qpos = reinterpret_cast<const float4*>(d_qpos4);
    a.qnrm = reinterpret_cast<const float4*>(d_qnrm4);
    a.grad = reinterpret_cast<const float4*>(d_grad_rad4);
    a.n = m->n; a.k = k; a.r_max = desc->r_max; a.filter = desc->filter;
    a.cone_k = desc->filter == PM_FILTER_CONE ? desc->cone_k : 1.0f;
    a.min_found = desc->min_found;
    a.qrec = P<BwdQuery>(m->qrec);
    a.vals = nullptr; a.cursor = nullptr; a.pair_cap = 0;
    a.nbr = nullptr; a.count_in = nullptr; a.order = nullptr;
    BwdBuffers b;
    b.vals[0] = P<uint32_t>(m->bvals); b.vals[1] = P<uint32_t>(m->bvals1);
    b.keys[0] = P<uint32_t>(m->bkeys0); b.keys[1] = P<uint32_t>(m->bkeys1);
    b.scratch = P<uint32_t>(m->bscratch);
    b.seg_start = P<uint32_t>(m->seg_start); b.seg_end = P<uint32_t>(m->seg_end);
    b.long_count = P<uint32_t>(m->blong); b.long_list = b.long_count + 1;
    b.acc = P<double>(m->acc);
    int nl = 0;
    for (uint32_t c = 0; c < nchunks; ++c) {
        const uint32_t q0 = c * chunk;
        const uint32_t nqc = nq ? ((nq - q0) < chunk ? (nq - q0) : chunk) : 0;
        // the chunk's queries in Hilbert order: the recomputed forward and the
        // adjoint's per-query pass walk them in it
        a.order = (sorted && nqc > 0) ? sort_queries(m, a.qpos + q0, nqc, st, &nl) : nullptr;
        if (recompute) {
            if (nqc > 0) {
                QueryOutputs out{P<float4>(m->rrad), P<uint32_t>(m->rnbr), P<float>(m->rr2), P<uint32_t>(m->rcnt)};
                QueryTuning t = tuning_of(m);
                t.stats = nullptr;
                nl += query_knn(view_of(m), params_of(desc), a.qpos + q0, a.qnrm + q0, a.order, nqc, out,
                                P<uint32_t>(m->counter), P<uint32_t>(m->fixq), t, st);
            }
            a.nbr = P<uint32_t>(m->rnbr);
            a.count_in = P<uint32_t>(m->rcnt);
        } else {
            a.nbr = d_nbr + (size_t)q0 * k;
            a.count_in = d_count ? d_count + q0 : nullptr;
        }
        nl += backward_chunk(a, q0, nqc, c == 0, c + 1 == nchunks, b, reinterpret_cast<float4*>(d_grad_pow4),
                             reinterpret_cast<float4*>(d_grad_pos4), st);
    }
    m->launches += (uint64_t)nl;
    return check_cuda(m, "pm_query_backward");
}

static pm_status icut_interp_run(pm_map* m, float r_max, const float4* qpos, const float4* qnrm, uint32_t nq,
                                 bool sorted, float4* out, cudaStream_t st, int* nl);

pm_status pm_gather_for(pm_map* m, const pm_query_desc* desc, const float* d_hit_pos4, const float* d_hit_nrm4,
                        const float* d_ray_dir4, const float* d_ray_origin4, const float* d_ray_influence4,
                        const float* d_clr_diffuse4, const uint32_t* d_idx_shading, uint32_t n, float* d_io_radiance4,
                        float* d_io_recip_dist, void* stream) {
    if (!m) return PM_ERR_INVALID;
    pm_status s = validate_desc(m, desc, true, true);
    if (s != PM_OK) return s;
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    const bool icut = desc->mode == PM_MODE_ICUT;
    if (icut && m->icut_gen != m->build_gen)
        return fail(m, PM_ERR_STATE, "PM_MODE_ICUT needs an illumination cut of the current tree (pm_icut_build)");
    if (n > kMaxQueries) return fail(m, PM_ERR_UNSUPPORTED, "n = %u exceeds 2^31 - 1 shading points", n);
    if (n > 0 && (!d_hit_pos4 || !d_hit_nrm4 || !d_ray_dir4 || !d_ray_influence4 || !d_io_radiance4))
        return fail(m, PM_ERR_INVALID, "hit positions, normals, ray directions, influences and radiance must be non-NULL");
    if (n > 0 && d_io_recip_dist && !d_ray_origin4)
        return fail(m, PM_ERR_INVALID, "ray origins are needed for the reciprocal-distance accumulator");
    const void* f4[] = {d_hit_pos4, d_hit_nrm4, d_ray_dir4, d_ray_origin4, d_ray_influence4, d_clr_diffuse4, d_io_radiance4};
    for (const void* p : f4)
        if (p && !aligned16(p)) return fail(m, PM_ERR_INVALID, "float4 arrays must be 16-byte aligned");
    if (n == 0 || m->n == 0) return PM_OK;   // nothing to gather (PhotonMap.cpp:239-240)
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    s = ensure_query_capacity(m, n, st);
    if (s != PM_OK) return s;
    if (m->gnrm.bytes < (size_t)n * sizeof(float4) || m->gest.bytes < (size_t)n * sizeof(float4)) {
        if (capturing(st)) return fail(m, PM_ERR_STATE, "gather storage must grow during stream capture");
        if ((s = buf_ensure(m, m->gnrm, (size_t)n * sizeof(float4), "gnrm")) != PM_OK) return s;
        if ((s = buf_ensure(m, m->gest, (size_t)n * sizeof(float4), "gest")) != PM_OK) return s;
    }
    const float4* hit = reinterpret_cast<const float4*>(d_hit_pos4);
    int nl = 0;
    if (icut) {
        // kernel_InterpolateIrradiance (GPU/photon_knn.cu:598-660): the cut
        // interpolated at the hit with the unflipped shading normal
        s = icut_interp_run(m, desc->r_max, hit, reinterpret_cast<const float4*>(d_hit_nrm4), n,
                            desc->order == PM_ORDER_SORTED, P<float4>(m->gest), st, &nl);
        if (s != PM_OK) return s;
    } else {
        nl += gather_normals(reinterpret_cast<const float4*>(d_hit_nrm4), reinterpret_cast<const float4*>(d_ray_dir4), n,
                             P<float4>(m->gnrm), st);
        const uint32_t* order = desc->order == PM_ORDER_SORTED ? sort_queries(m, hit, n, st, &nl) : nullptr;
        QueryParams qp = params_of(desc);
        if (!d_clr_diffuse4) qp.min_found = 0;   // photon visualisation keeps every estimate (GPU/photon_knn.cu:515-519)
        QueryOutputs out{P<float4>(m->gest), nullptr, nullptr, nullptr};
        QueryTuning t = tuning_of(m);
        t.stats = nullptr;
        nl += query_knn(view_of(m), qp, hit, P<float4>(m->gnrm), order, n, out, P<uint32_t>(m->counter),
                        P<uint32_t>(m->fixq), t, st);
    }
    nl += gather_accumulate(P<float4>(m->gest), hit, reinterpret_cast<const float4*>(d_ray_origin4),
                            reinterpret_cast<const float4*>(d_ray_influence4),
                            reinterpret_cast<const float4*>(d_clr_diffuse4), d_idx_shading, n,
                            reinterpret_cast<float4*>(d_io_radiance4), d_io_recip_dist, st);
    m->launches += (uint64_t)nl;
    return check_cuda(m, "pm_gather_for");
}

// ---- illumination cuts -----------------------------------------------------

static IcutBuffers icut_of(pm_map* m) {
    IcutBuffers b;
    b.pslot = P<uint32_t>(m->ic_pslot); b.level = P<uint32_t>(m->ic_level); b.range = P<uint2>(m->ic_range);
    b.center = P<float4>(m->ic_center); b.normal = P<float4>(m->ic_normal); b.est = P<float4>(m->ic_est);
    b.exact = P<float4>(m->ic_exact); b.coarse = P<uint32_t>(m->ic_coarse); b.fin = P<uint32_t>(m->ic_fin);
    b.work[0] = P<uint32_t>(m->ic_work0); b.work[1] = P<uint32_t>(m->ic_work1);
    b.acc = P<unsigned long long>(m->ic_acc);
    b.ibox = P<float4>(m->ic_ibox);
    return b;
}

// Slot records of the current tree (levels, photon ranges, centres); reads
// the node count from the device, so it synchronises the stream.
static pm_status icut_prepare_now(pm_map* m, cudaStream_t st) {
    if (m->icut_prep_gen == m->build_gen) return PM_OK;
    if (capturing(st)) return fail(m, PM_ERR_STATE, "illumination cuts cannot be prepared during stream capture");
    MapHeader h;
    if (cudaMemcpyAsync(&h, m->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return check_cuda(m, "pm_icut: node count");
    const uint32_t nodes = h.num_nodes;
    const size_t ns = 2 * ((size_t)nodes + 1);
    if (ns > (1u << 27)) return fail(m, PM_ERR_UNSUPPORTED, "illumination cuts support at most 2^27 tree slots");
    pm_status s;
#define ENSURE(buf, bytes) if ((s = buf_ensure(m, m->buf, (bytes), #buf)) != PM_OK) return s
    ENSURE(ic_pslot, ((size_t)nodes + 2) * sizeof(uint32_t));
    ENSURE(ic_level, ns * sizeof(uint32_t));
    ENSURE(ic_range, ns * sizeof(uint2));
    ENSURE(ic_center, ns * sizeof(float4));
    ENSURE(ic_normal, ns * sizeof(float4));
    ENSURE(ic_est, ns * sizeof(float4));
    ENSURE(ic_exact, ns * sizeof(float4));
    ENSURE(ic_coarse, ns * sizeof(uint32_t));
    ENSURE(ic_fin, ns * sizeof(uint32_t));
    ENSURE(ic_work0, ns * sizeof(uint32_t));
    ENSURE(ic_work1, ns * sizeof(uint32_t));
    ENSURE(ic_acc, 8 * sizeof(unsigned long long));
    ENSURE(ic_ibox, 2 * ns * sizeof(float4));
#undef ENSURE
    m->launches += (uint64_t)icut_prepare(view_of(m), nodes, icut_of(m), st);
    s = check_cuda(m, "pm_icut: slot records");
    if (s != PM_OK) return s;
    m->icut_slots = (uint32_t)ns;
    m->icut_prep_gen = m->build_gen;
    return PM_OK;
}

static pm_status icut_interp_run(pm_map* m, float r_max, const float4* qpos, const float4* qnrm, uint32_t nq,
                                 bool sorted, float4* out, cudaStream_t st, int* nl) {
    pm_status s = ensure_query_capacity(m, nq, st);
    if (s != PM_OK) return s;
    // Morton order: the interpolation is a thread per query (see k_query_order)
    const uint32_t* order = sorted ? sort_queries(m, qpos, nq, st, nl, false) : nullptr;
    *nl += icut_interpolate(view_of(m), icut_of(m), qpos, qnrm, order, nq, r_max * r_max, out, st);
    return PM_OK;
}

pm_status pm_icut_build(pm_map* m, const pm_icut_desc* cut, const pm_query_desc* node_query,
                        const float* d_node_normals4, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (!cut) return fail(m, PM_ERR_INVALID, "cut descriptor is NULL");
    pm_status s = validate_desc(m, node_query, false);
    if (s != PM_OK) return s;
    if (cut->refine_iters > 64) return fail(m, PM_ERR_INVALID, "refine_iters must be at most 64");
    if (!(cut->accuracy >= 0.0f) || !std::isfinite(cut->accuracy))
        return fail(m, PM_ERR_INVALID, "accuracy must be finite and >= 0");
    if (d_node_normals4 && !aligned16(d_node_normals4))
        return fail(m, PM_ERR_INVALID, "node normals must be 16-byte aligned");
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    s = icut_prepare_now(m, st);
    if (s != PM_OK) return s;
    const uint32_t ns = m->icut_slots;
    const MapView v = view_of(m);
    const IcutBuffers b = icut_of(m);
    const IcutParams p{cut->use_leafs != 0, cut->level_emin, cut->refine_iters, cut->accuracy};
    int nl = icut_normals(v, ns, reinterpret_cast<const float4*>(d_node_normals4), b, st);
    nl += icut_coarse(v, ns, p, b, st);
    // irradiance at every slot centre with the slot's normal (PhotonMap.cpp:371-384)
    if (node_query->mode == PM_MODE_ZHOU_COMPAT) {
        s = compat_run(m, node_query, reinterpret_cast<const float*>(b.center), reinterpret_cast<const float*>(b.normal),
                       ns, nullptr, reinterpret_cast<float*>(b.exact), nullptr, nullptr, st);
        if (s != PM_OK) return s;
    } else {
        s = ensure_query_capacity(m, ns, st);
        if (s != PM_OK) return s;
        const uint32_t* order = node_query->order == PM_ORDER_SORTED ? sort_queries(m, b.center, ns, st, &nl) : nullptr;
        QueryOutputs out{b.exact, nullptr, nullptr, nullptr};
        QueryTuning t = tuning_of(m);
        t.stats = nullptr;
        nl += query_knn(v, params_of(node_query), b.center, b.normal, order, ns, out, P<uint32_t>(m->counter),
                        P<uint32_t>(m->fixq), t, st);
    }
    nl += icut_final(v, ns, p, b, st);
    m->launches += (uint64_t)nl;
    s = check_cuda(m, "pm_icut_build");
    if (s != PM_OK) return s;
    m->icut_gen = m->build_gen;
    return PM_OK;
}

pm_status pm_icut_slot_count(pm_map* m, uint32_t* count) {
    if (!m || !count) return fail(m, PM_ERR_INVALID, "count is NULL");
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    MapHeader h;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&h, m->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
        return check_cuda(m, "pm_icut_slot_count");
    *count = 2 * (h.num_nodes + 1);
    return PM_OK;
}

pm_status pm_icut_node_centers(pm_map* m, float* d_centers4, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (!d_centers4 || !aligned16(d_centers4)) return fail(m, PM_ERR_INVALID, "centres must be a 16-byte aligned array");
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    pm_status s = icut_prepare_now(m, st);
    if (s != PM_OK) return s;
    cudaMemcpyAsync(d_centers4, m->ic_center.ptr, (size_t)m->icut_slots * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    return check_cuda(m, "pm_icut_node_centers");
}

pm_status pm_icut_interpolate(pm_map* m, float r_max, const float* d_qpos4, const float* d_qnrm4, uint32_t nq,
                              float* d_irr4, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (!(r_max > 0.0f) || !std::isfinite(r_max))
        return fail(m, PM_ERR_INVALID, "r_max must be finite and > 0 (got %g)", (double)r_max);
    if (nq > kMaxQueries) return fail(m, PM_ERR_UNSUPPORTED, "nq = %u exceeds 2^31 - 1 queries", nq);
    if (nq > 0 && (!d_qpos4 || !d_qnrm4 || !d_irr4))
        return fail(m, PM_ERR_INVALID, "query positions, normals and output must be non-NULL");
    if (nq > 0 && (!aligned16(d_qpos4) || !aligned16(d_qnrm4) || !aligned16(d_irr4)))
        return fail(m, PM_ERR_INVALID, "query and output arrays must be 16-byte aligned");
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    if (m->icut_gen != m->build_gen)
        return fail(m, PM_ERR_STATE, "no illumination cut for the current tree (call pm_icut_build)");
    if (nq == 0) return PM_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int nl = 0;
    pm_status s = icut_interp_run(m, r_max, reinterpret_cast<const float4*>(d_qpos4),
                                  reinterpret_cast<const float4*>(d_qnrm4), nq, true, reinterpret_cast<float4*>(d_irr4),
                                  st, &nl);
    if (s != PM_OK) return s;
    m->launches += (uint64_t)nl;
    return check_cuda(m, "pm_icut_interpolate");
}

pm_status pm_icut_export(pm_map* m, uint32_t max_slots, uint32_t* h_coarse, uint32_t* h_final, uint32_t* h_level,
                         float* h_center4, float* h_normal4, float* h_est4, float* h_exact4) {
    if (!m) return PM_ERR_INVALID;
    if (!m->built || m->icut_gen != m->build_gen)
        return fail(m, PM_ERR_STATE, "no illumination cut for the current tree (call pm_icut_build)");
    const uint32_t ns = m->icut_slots;
    if (max_slots < ns) return fail(m, PM_ERR_INVALID, "need room for %u slots", ns);
    if (cudaDeviceSynchronize() != cudaSuccess) return check_cuda(m, "pm_icut_export");
    struct Out { void* dst; const DevBuf* src; size_t elem; } outs[] = {
        {h_coarse, &m->ic_coarse, 4}, {h_final, &m->ic_fin, 4}, {h_level, &m->ic_level, 4},
        {h_center4, &m->ic_center, 16}, {h_normal4, &m->ic_normal, 16}, {h_est4, &m->ic_est, 16},
        {h_exact4, &m->ic_exact, 16}};
    for (const Out& o : outs)
        if (o.dst && cudaMemcpy(o.dst, o.src->ptr, (size_t)ns * o.elem, cudaMemcpyDeviceToHost) != cudaSuccess)
            return check_cuda(m, "pm_icut_export");
    return PM_OK;
}

pm_status pm_scale_flux(pm_map* m, float scale, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (!std::isfinite(scale)) return fail(m, PM_ERR_INVALID, "scale must be finite");
    if (!m->built && m->merged_n == 0) return fail(m, PM_ERR_STATE, "no photons to scale (nothing merged or built)");
    if (!m->built) {
        m->launches += (uint64_t)scale_rgb(P<float4>(m->mpow), m->merged_n, scale, reinterpret_cast<cudaStream_t>(stream));
        return check_cuda(m, "pm_scale_flux");
    }
    scale_flux(P<float4>(m->pow), m->n, scale, P<MapHeader>(m->hdr), reinterpret_cast<cudaStream_t>(stream));
    m->launches += 1;
    m->launches += (uint64_t)scale_rgb(P<float4>(m->mpow), m->merged_n, scale, reinterpret_cast<cudaStream_t>(stream));
    return check_cuda(m, "pm_scale_flux");
}

pm_status pm_compute_query_radii(pm_map* m, const pm_query_desc* desc, const float* d_qpos4, uint32_t nq,
                                 float* d_radii, void* stream) {
    if (!m) return PM_ERR_INVALID;
    pm_status s = validate_desc(m, desc, false);
    if (s != PM_OK) return s;
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    if (nq > kMaxQueries) return fail(m, PM_ERR_UNSUPPORTED, "nq = %u exceeds 2^31 - 1 queries", nq);
    if (nq > 0 && (!d_qpos4 || !d_radii)) return fail(m, PM_ERR_INVALID, "query positions and radii must be non-NULL");
    if (nq > 0 && !aligned16(d_qpos4)) return fail(m, PM_ERR_INVALID, "query positions must be 16-byte aligned");
    return compat_run(m, desc, d_qpos4, d_qpos4, nq, d_radii, nullptr, nullptr, nullptr,
                      reinterpret_cast<cudaStream_t>(stream));
}

pm_status pm_get_info(pm_map* m, pm_map_info* info, void* stream) {
    if (!m || !info) return fail(m, PM_ERR_INVALID, "info is NULL");
    std::memset(info, 0, sizeof(*info));
    info->leaf_size = m->leaf_size;
    info->num_photons = m->n;
    if (!m->built) return PM_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    MapHeader h;
    if (cudaMemcpyAsync(&h, m->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return check_cuda(m, "pm_get_info");
    info->num_nodes = h.num_nodes;
    info->device_errors = h.errors;
    for (int a = 0; a < 3; ++a) { info->bounds_min[a] = h.lo[a]; info->bounds_max[a] = h.hi[a]; }
    info->max_power = h.max_power;
    info->launches = m->launches;
    return PM_OK;
}

pm_status pm_set_profiling(pm_map* m, int enable) {
    if (!m) return PM_ERR_INVALID;
    if (enable) {
        for (cudaEvent_t& e : m->ev)
            if (!e && cudaEventCreate(&e) != cudaSuccess) return check_cuda(m, "pm_set_profiling");
    }
    if (enable >= 2) {
        pm_status s = buf_ensure(m, m->stats, 16 * sizeof(unsigned long long), "stats");
        if (s != PM_OK) return s;
    }
    m->profiling = enable != 0;
    m->profile_level = enable;
    return PM_OK;
}

pm_status pm_query_stats(pm_map* m, uint64_t* out, uint32_t count) {
    if (!m || !out) return fail(m, PM_ERR_INVALID, "stats output is NULL");
    if (!m->stats.ptr || m->profile_level < 2) return fail(m, PM_ERR_STATE, "enable profiling level 2 first");
    const uint32_t c = count < 8 ? count : 8;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(out, m->stats.ptr, c * sizeof(uint64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return check_cuda(m, "pm_query_stats");
    return PM_OK;
}

pm_status pm_last_timings(pm_map* m, pm_timings* out) {
    if (!m || !out) return fail(m, PM_ERR_INVALID, "timings output is NULL");
    std::memset(out, 0, sizeof(*out));
    out->build_launches = m->build_launches;
    out->query_launches = m->query_launches;
    if (m->have_build_ev) {
        if (cudaEventSynchronize(m->ev[2]) != cudaSuccess) return check_cuda(m, "pm_last_timings");
        cudaEventElapsedTime(&out->build_ms, m->ev[0], m->ev[2]);
        cudaEventElapsedTime(&out->build_sort_ms, m->ev[0], m->ev[1]);
    }
    if (m->have_query_ev) {
        if (cudaEventSynchronize(m->ev[5]) != cudaSuccess) return check_cuda(m, "pm_last_timings");
        cudaEventElapsedTime(&out->query_ms, m->ev[3], m->ev[5]);
        cudaEventElapsedTime(&out->query_sort_ms, m->ev[3], m->ev[4]);
        cudaEventElapsedTime(&out->query_kernel_ms, m->ev[4], m->ev[5]);
    }
    return check_cuda(m, "pm_last_timings");
}

pm_status pm_clear_errors(pm_map* m, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (!m->hdr.ptr) return PM_OK;
    cudaMemsetAsync(&P<MapHeader>(m->hdr)->errors, 0, sizeof(uint32_t), reinterpret_cast<cudaStream_t>(stream));
    return check_cuda(m, "pm_clear_errors");
}

pm_status pm_export_tree(pm_map* m, uint32_t* host_nodes, uint32_t max_nodes, float* host_pos4, float* host_pow4,
                         uint32_t max_photons) {
    if (!m) return PM_ERR_INVALID;
    if (!m->built) return fail(m, PM_ERR_STATE, "no photon map has been built");
    if (cudaDeviceSynchronize() != cudaSuccess) return check_cuda(m, "pm_export_tree");
    MapHeader h;
    if (cudaMemcpy(&h, m->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return check_cuda(m, "pm_export_tree");
    const uint32_t total_nodes = h.num_nodes + 1;
    if (host_nodes) {
        if (max_nodes < total_nodes) return fail(m, PM_ERR_INVALID, "need room for %u nodes", total_nodes);
        if (cudaMemcpy(host_nodes, m->nodes.ptr, (size_t)total_nodes * sizeof(Node), cudaMemcpyDeviceToHost) != cudaSuccess)
            return check_cuda(m, "pm_export_tree");
    }
    if (host_pos4 || host_pow4) {
        if (max_photons < m->n) return fail(m, PM_ERR_INVALID, "need room for %u photons", m->n);
        if (host_pos4 && m->n &&
            cudaMemcpy(host_pos4, m->pos.ptr, (size_t)m->n * sizeof(float4), cudaMemcpyDeviceToHost) != cudaSuccess)
            return check_cuda(m, "pm_export_tree");
        if (host_pow4 && m->n &&
            cudaMemcpy(host_pow4, m->pow.ptr, (size_t)m->n * sizeof(float4), cudaMemcpyDeviceToHost) != cudaSuccess)
            return check_cuda(m, "pm_export_tree");
    }
    return PM_OK;
}

}  // extern "C"
// ---------------------------------------------------------------------------
// pm_query_noalloc: the query with its scratch in a fixed array.
//
// Some callers cannot allocate device memory when they query: cudaMalloc and
// cudaFree synchronise the whole device, which stalls a render loop, and some
// host applications hand the engine a fixed memory budget up front and let
// nothing grow afterwards.  This entry point runs the same kernels as
// pm_query, but the scratch they need beyond the caller's inputs and outputs
// (query Hilbert keys, radix-sort histograms, the list of queries re-evaluated
// with FP64 distances, the work counters) is carved from
// one file-scope device array of a fixed size.  The map itself must already
// be built.  Nothing here calls cudaMalloc, cudaFree or any allocating
// library routine.
//
// The array is shared by every call on every handle.  Each call rewrites all
// of it that it reads (the keys, the histograms, the fix list) and query_knn
// clears the counters on the stream before the kernel starts, so one call's leftovers
// never leak into the next; calls that overlap on the GPU race.
namespace {

constexpr uint32_t kNoallocMaxQ = PM_NOALLOC_MAX_QUERIES;
constexpr size_t kNoallocSortWords = 33024;   // >= sort_scratch_words(kNoallocMaxQ) = 33024, checked at set-up
constexpr size_t kNoallocAlign = 256;
constexpr size_t noalloc_round(size_t b) { return (b + kNoallocAlign - 1) / kNoallocAlign * kNoallocAlign; }
// The single-map query sorts 32-bit Hilbert keys: 4 bytes per query for each
// key and value buffer.
constexpr size_t kNoallocKeys0 = 0;
constexpr size_t kNoallocKeys1 = kNoallocKeys0 + noalloc_round((size_t)kNoallocMaxQ * sizeof(uint32_t));
constexpr size_t kNoallocVals0 = kNoallocKeys1 + noalloc_round((size_t)kNoallocMaxQ * sizeof(uint32_t));
constexpr size_t kNoallocVals1 = kNoallocVals0 + noalloc_round((size_t)kNoallocMaxQ * sizeof(uint32_t));
constexpr size_t kNoallocSort = kNoallocVals1 + noalloc_round((size_t)kNoallocMaxQ * sizeof(uint32_t));
constexpr size_t kNoallocFix = kNoallocSort + noalloc_round(kNoallocSortWords * sizeof(uint32_t));
constexpr size_t kNoallocCounter = kNoallocFix + noalloc_round((size_t)kNoallocMaxQ * sizeof(uint32_t));
constexpr size_t kNoallocBytes = kNoallocCounter + kNoallocAlign;

// In host code this name is only a host-side handle for the runtime: its
// device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of the scratch array on the current device (looked up on
// the first call per device, with that device current).  The lookup may load
// the module, which must not happen inside a stream capture: a first call on
// a capturing stream is refused with PM_ERR_STATE before any runtime call
// that could invalidate the capture.  The cached address is never refreshed;
// after cudaDeviceReset it no longer names the array (the header says so).
pm_status noalloc_scratch(pm_map* m, cudaStream_t st, unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return check_cuda(m, "pm_query_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kNoallocMaxDevices)
        return fail(m, PM_ERR_UNSUPPORTED, "pm_query_noalloc supports device ordinals below %d", kNoallocMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        if (capturing(st))
            return fail(m, PM_ERR_STATE, "the first pm_query_noalloc call on a device must come before any stream "
                                         "capture (it looks up the scratch array's address)");
        if (sort_scratch_words(kNoallocMaxQ) > kNoallocSortWords)
            return fail(m, PM_ERR_STATE, "pm_query_noalloc: sort scratch of the fixed array is too small");
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(m, PM_ERR_CUDA, "pm_query_noalloc: cudaGetSymbolAddress of the scratch array failed: %s",
                        cudaGetErrorString(e));
        }
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return PM_OK;
}

}  // namespace

extern "C" pm_status pm_query_noalloc(pm_map* m, const pm_query_desc* desc, const float* d_qpos4,
                                      const float* d_qnrm4, uint32_t nq, float* d_rad4, uint32_t* d_nbr, float* d_r2,
                                      uint32_t* d_count, void* stream) {
    pm_status s = query_common(m, desc, d_qpos4, d_qnrm4, nq, d_rad4, false);
    if (s != PM_OK) return s;
    if (desc->mode == PM_MODE_ZHOU_COMPAT)
        return fail(m, PM_ERR_UNSUPPORTED, "pm_query_noalloc supports PM_MODE_EXACT only");
    if (nq > kNoallocMaxQ)
        return fail(m, PM_ERR_INVALID, "nq = %u exceeds PM_NOALLOC_MAX_QUERIES = %u; split the queries", nq,
                    kNoallocMaxQ);
    if (nq == 0) return PM_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    s = noalloc_scratch(m, st, &base);
    if (s != PM_OK) return s;
    const float4* qpos = reinterpret_cast<const float4*>(d_qpos4);
    int nl = 0;
    const uint32_t* order = nullptr;
    if (desc->order == PM_ORDER_SORTED) {
        uint32_t* keys[2] = {reinterpret_cast<uint32_t*>(base + kNoallocKeys0),
                             reinterpret_cast<uint32_t*>(base + kNoallocKeys1)};
        uint32_t* vals[2] = {reinterpret_cast<uint32_t*>(base + kNoallocVals0),
                             reinterpret_cast<uint32_t*>(base + kNoallocVals1)};
        nl += query_order_keys(qpos, nq, P<MapHeader>(m->hdr), keys[0], vals[0], st);
        const int cur = radix_sort_pairs32(keys, vals, nq, kQueryKeyBits, reinterpret_cast<uint32_t*>(base + kNoallocSort),
                                           st, &nl);
        order = vals[cur];
    }
    QueryTuning t = tuning_of(m);
    t.stats = nullptr;
    QueryOutputs out{reinterpret_cast<float4*>(d_rad4), d_nbr, d_r2, d_count};
    nl += query_knn(view_of(m), params_of(desc), qpos, reinterpret_cast<const float4*>(d_qnrm4), order, nq, out,
                    reinterpret_cast<uint32_t*>(base + kNoallocCounter), reinterpret_cast<uint32_t*>(base + kNoallocFix),
                    t, st);
    // no phase events and no traversal counters here: pm_last_timings then
    // reports this call's launch count and no query times
    m->have_query_ev = false;
    m->query_launches = (uint32_t)nl;
    m->launches += (uint64_t)nl;
    return check_cuda(m, "pm_query_noalloc");
}

// ---------------------------------------------------------------------------
// Batches of photon maps (no counterpart in the reference, which builds and
// gathers one map per call).  A batch owns one pm_map for its combined
// storage plus the per-map tables; see pm_batch.cu for the device side.
struct pm_batch {
    pm_map* m = nullptr;
    uint32_t num_maps = 0;
    uint32_t total_photons = 0;
    bool built = false;
    int format = PM_PHOTONS_PACKED;
    DevBuf ph_off, q_off, bq, geom, acc;
    uint32_t cap_maps = 0;
    std::vector<uint32_t> h_ph_off;   // host copy of the built photon offsets
    // CUDA graph of build + query
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t query_launches = 0;
};

namespace {

pm_status batch_fail(pm_batch* b, pm_status s, const char* msg) {
    if (b && b->m) fail(b->m, s, "%s", msg);
    return s;
}

pm_status batch_tables(pm_batch* b, uint32_t maps) {
    if (maps <= b->cap_maps && b->ph_off.ptr) return PM_OK;
    pm_map* m = b->m;
    pm_status s;
    if ((s = buf_ensure(m, b->ph_off, (maps + 1) * sizeof(uint32_t), "batch photon offsets")) != PM_OK) return s;
    if ((s = buf_ensure(m, b->q_off, (maps + 1) * sizeof(uint32_t), "batch query offsets")) != PM_OK) return s;
    if ((s = buf_ensure(m, b->bq, maps * sizeof(BatchQuery), "batch query table")) != PM_OK) return s;
    if ((s = buf_ensure(m, b->geom, maps * sizeof(BatchGeom), "batch geometry")) != PM_OK) return s;
    if ((s = buf_ensure(m, b->acc, maps * 8 * sizeof(uint32_t), "batch bounds")) != PM_OK) return s;
    b->cap_maps = maps;
    return PM_OK;
}

// Validates and uploads the photon offsets (synchronously: tables are small
// and this runs outside any capture).
pm_status batch_upload_photons(pm_batch* b, const uint32_t* offsets, uint32_t maps) {
    if (!offsets) return batch_fail(b, PM_ERR_INVALID, "photon offsets are NULL");
    if (maps == 0 || maps > 65536) return batch_fail(b, PM_ERR_INVALID, "a batch holds 1 to 65536 maps");
    if (offsets[0] != 0) return batch_fail(b, PM_ERR_INVALID, "photon offsets must start at 0");
    for (uint32_t i = 0; i < maps; ++i)
        if (offsets[i + 1] < offsets[i]) return batch_fail(b, PM_ERR_INVALID, "photon offsets must not decrease");
    if (offsets[maps] > 0x7fffffffu) return batch_fail(b, PM_ERR_UNSUPPORTED, "more than 2^31 - 1 photons in a batch");
    pm_status s = batch_tables(b, maps);
    if (s != PM_OK) return s;
    if (cudaMemcpy(b->ph_off.ptr, offsets, (maps + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return check_cuda(b->m, "batch photon offsets");
    b->h_ph_off.assign(offsets, offsets + maps + 1);
    return PM_OK;
}

pm_status batch_upload_queries(pm_batch* b, const pm_query_desc* descs, const uint32_t* offsets, uint32_t* kmax_out,
                               uint64_t* nbr_total) {
    const uint32_t maps = b->num_maps;
    if (!descs || !offsets) return batch_fail(b, PM_ERR_INVALID, "query descriptors or offsets are NULL");
    if (offsets[0] != 0) return batch_fail(b, PM_ERR_INVALID, "query offsets must start at 0");
    std::vector<BatchQuery> t(maps);
    uint32_t kmax = 1;
    uint64_t nbr = 0;
    for (uint32_t i = 0; i < maps; ++i) {
        pm_status s = validate_desc(b->m, &descs[i], true);
        if (s != PM_OK) return s;
        if (offsets[i + 1] < offsets[i]) return batch_fail(b, PM_ERR_INVALID, "query offsets must not decrease");
        BatchQuery& q = t[i];
        q.q_off = offsets[i];
        q.q_n = offsets[i + 1] - offsets[i];
        q.ph_off = b->h_ph_off[i];
        q.ph_n = b->h_ph_off[i + 1] - b->h_ph_off[i];
        q.nbr_off = nbr;
        q.k = descs[i].k;
        q.min_found = descs[i].min_found;
        q.rmax = descs[i].r_max;
        q.r2max = descs[i].r_max * descs[i].r_max;
        q.filter = descs[i].filter;
        q.cone_k = descs[i].filter == PM_FILTER_CONE ? descs[i].cone_k : 1.0f;
        q.norm_c = filter_norm_const(q.filter, q.cone_k);
        nbr += (uint64_t)q.q_n * q.k;
        kmax = q.k > kmax ? q.k : kmax;
    }
    if (cudaMemcpy(b->bq.ptr, t.data(), maps * sizeof(BatchQuery), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->q_off.ptr, offsets, (maps + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return check_cuda(b->m, "batch query tables");
    *kmax_out = kmax;
    *nbr_total = nbr;
    return PM_OK;
}

// The device work of a batch build (tables already uploaded, storage sized).
pm_status batch_build_device(pm_batch* b, const float* d_pos4, const float* d_pow4, int format, cudaStream_t st) {
    pm_map* m = b->m;
    const uint32_t n = b->total_photons, maps = b->num_maps;
    BuildBuffers bb;
    bb.keys[0] = P<uint64_t>(m->keys0); bb.keys[1] = P<uint64_t>(m->keys1);
    bb.vals[0] = P<uint32_t>(m->vals0); bb.vals[1] = P<uint32_t>(m->vals1);
    bb.scratch = P<uint32_t>(m->scratch);
    bb.kfirst = P<uint32_t>(m->kfirst); bb.klast = P<uint32_t>(m->klast); bb.ksplit = P<uint32_t>(m->ksplit);
    bb.kkeep = P<uint32_t>(m->kkeep); bb.krank = P<uint32_t>(m->krank);
    bb.parent = P<uint32_t>(m->parent); bb.arrive = P<uint32_t>(m->arrive); bb.nleaf = P<uint32_t>(m->nleaf);
    bb.partials = P<uint32_t>(m->partials); bb.num_partials = 1184;
    const float4* pos = reinterpret_cast<const float4*>(d_pos4);
    const float4* pw = reinterpret_cast<const float4*>(d_pow4);
    int nl = batch_bounds_and_keys(pos, pw, P<uint32_t>(b->ph_off), maps, n, P<uint32_t>(b->acc),
                                   P<BatchGeom>(b->geom), P<MapHeader>(m->hdr), bb.keys[0], bb.vals[0], st);
    uint64_t* keys[2] = {bb.keys[0], bb.keys[1]};
    uint32_t* vals[2] = {bb.vals[0], bb.vals[1]};
    const SortGather g{pos, pw, format, P<float4>(m->pos), P<float4>(m->pow), P<uint32_t>(m->inv)};
    const int cur = n > 1 ? radix_sort_pairs(keys, vals, n, kMortonBits + map_id_bits(maps), bb.scratch, st, &nl, &g) : 0;
    nl += build_from_sorted(pos, pw, n, format, m->leaf_size, keys[cur], vals[cur], P<float4>(m->pos),
                            P<float4>(m->pow), P<uint32_t>(m->inv), P<Node>(m->nodes), P<MapHeader>(m->hdr), bb, st,
                            n > 1);
    nl += batch_roots(P<uint32_t>(b->ph_off), maps, n, m->leaf_size, P<float4>(m->pos), P<Node>(m->nodes), bb,
                      P<BatchGeom>(b->geom), st);
    nl += batch_wide(n, maps, P<Node>(m->nodes), P<uint32_t>(m->parent), P<MapHeader>(m->hdr), P<uint32_t>(m->rootmark),
                     wide_of(m), P<BatchGeom>(b->geom), st);
    m->launches += (uint64_t)nl;
    m->build_launches = (uint32_t)nl;
    return check_cuda(m, "pm_batch_build");
}

pm_status batch_query_device(pm_batch* b, uint32_t kmax, const float* d_qpos4, const float* d_qnrm4, uint32_t nq,
                             float* d_rad4, uint32_t* d_nbr, float* d_r2, uint32_t* d_count, cudaStream_t st) {
    pm_map* m = b->m;
    if (nq == 0) return PM_OK;
    const float4* qpos = reinterpret_cast<const float4*>(d_qpos4);
    int nl = batch_query_keys(qpos, P<uint32_t>(b->q_off), b->num_maps, nq, P<BatchGeom>(b->geom),
                              P<uint64_t>(m->qkeys0), P<uint32_t>(m->qvals0), st);
    uint64_t* keys[2] = {P<uint64_t>(m->qkeys0), P<uint64_t>(m->qkeys1)};
    uint32_t* vals[2] = {P<uint32_t>(m->qvals0), P<uint32_t>(m->qvals1)};
    const int cur = nq > 1 ? radix_sort_pairs(keys, vals, nq, kBatchQueryMapShift + map_id_bits(b->num_maps),
                                              P<uint32_t>(m->qscratch), st, &nl)
                           : 0;
    QueryOutputs out{reinterpret_cast<float4*>(d_rad4), d_nbr, d_r2, d_count};
    QueryTuning t = tuning_of(m);
    t.stats = nullptr;
    nl += query_knn_batch(view_of(m), P<BatchQuery>(b->bq), P<BatchGeom>(b->geom), kmax, qpos,
                          reinterpret_cast<const float4*>(d_qnrm4), vals[cur], keys[cur], nq, out, P<uint32_t>(m->counter),
                          P<uint32_t>(m->fixq), t, st);
    m->launches += (uint64_t)nl;
    b->query_launches = (uint32_t)nl;
    return check_cuda(m, "pm_batch_query");
}

pm_status batch_check_query_args(pm_batch* b, const uint32_t* offsets, const float* d_qpos4, const float* d_qnrm4,
                                 float* d_rad4, uint32_t* nq_out) {
    if (!b->built) return batch_fail(b, PM_ERR_STATE, "the batch has not been built");
    if (!offsets) return batch_fail(b, PM_ERR_INVALID, "query offsets are NULL");
    const uint32_t nq = offsets[b->num_maps];
    if (nq > kMaxQueries) return batch_fail(b, PM_ERR_UNSUPPORTED, "more than 2^31 - 1 queries in a batch");
    if (nq > 0 && (!d_qpos4 || !d_qnrm4 || !d_rad4))
        return batch_fail(b, PM_ERR_INVALID, "query positions, normals and radiance output must be non-NULL");
    if (nq > 0 && (!aligned16(d_qpos4) || !aligned16(d_qnrm4) || !aligned16(d_rad4)))
        return batch_fail(b, PM_ERR_INVALID, "query and radiance arrays must be 16-byte aligned");
    *nq_out = nq;
    return PM_OK;
}

pm_status batch_prepare_build(pm_batch* b, const float* d_pos4, const float* d_pow4, const uint32_t* photon_offsets,
                              uint32_t num_maps, int format) {
    if (format != PM_PHOTONS_REFERENCE && format != PM_PHOTONS_PACKED)
        return batch_fail(b, PM_ERR_INVALID, "unknown photon format");
    pm_status s = batch_upload_photons(b, photon_offsets, num_maps);
    if (s != PM_OK) return s;
    const uint32_t n = photon_offsets[num_maps];
    if (n > 0 && (!d_pos4 || !d_pow4)) return batch_fail(b, PM_ERR_INVALID, "photon arrays must be non-NULL");
    if (n > 0 && (!aligned16(d_pos4) || !aligned16(d_pow4)))
        return batch_fail(b, PM_ERR_INVALID, "photon arrays must be 16-byte aligned");
    s = ensure_photon_capacity(b->m, n, nullptr);
    if (s != PM_OK) return s;
    b->num_maps = num_maps;
    b->total_photons = n;
    b->format = format;
    return PM_OK;
}

}  // namespace

extern "C" {

pm_status pm_batch_create(pm_batch** out) {
    if (!out) return PM_ERR_INVALID;
    *out = nullptr;
    pm_batch* b = new (std::nothrow) pm_batch();
    if (!b) return PM_ERR_OOM;
    pm_status s = pm_create(&b->m, 0, nullptr, nullptr, 1.0f);
    if (s != PM_OK) { delete b; return s; }
    *out = b;
    return PM_OK;
}

pm_status pm_batch_destroy(pm_batch* b) {
    if (!b) return PM_ERR_INVALID;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    DevBuf* all[] = {&b->ph_off, &b->q_off, &b->bq, &b->geom, &b->acc};
    for (DevBuf* x : all) buf_free(b->m, *x);
    pm_destroy(b->m);
    delete b;
    return PM_OK;
}

pm_status pm_batch_set_tuning(pm_batch* b, uint32_t leaf_size, int warps_per_block, int rounds_per_chunk, int wide) {
    if (!b) return PM_ERR_INVALID;
    return pm_set_tuning(b->m, leaf_size, warps_per_block, rounds_per_chunk, 1, wide ? PM_KBUF_WIDE : PM_KBUF_GROUP);
}

pm_status pm_batch_build(pm_batch* b, const float* d_pos4, const float* d_pow4, const uint32_t* photon_offsets,
                         uint32_t num_maps, int format, void* stream) {
    if (!b) return PM_ERR_INVALID;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (capturing(st)) return batch_fail(b, PM_ERR_STATE, "use pm_batch_capture to record a batch in a graph");
    pm_status s = batch_prepare_build(b, d_pos4, d_pow4, photon_offsets, num_maps, format);
    if (s != PM_OK) return s;
    s = batch_build_device(b, d_pos4, d_pow4, format, st);
    if (s != PM_OK) return s;
    b->m->n = b->total_photons;
    b->m->built = true;
    b->built = true;
    return PM_OK;
}

pm_status pm_batch_query(pm_batch* b, const pm_query_desc* descs, const float* d_qpos4, const float* d_qnrm4,
                         const uint32_t* query_offsets, float* d_rad4, uint32_t* d_nbr, float* d_r2, uint32_t* d_count,
                         void* stream) {
    if (!b) return PM_ERR_INVALID;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (capturing(st)) return batch_fail(b, PM_ERR_STATE, "use pm_batch_capture to record a batch in a graph");
    uint32_t nq = 0, kmax = 1;
    uint64_t nbr_total = 0;
    pm_status s = batch_check_query_args(b, query_offsets, d_qpos4, d_qnrm4, d_rad4, &nq);
    if (s != PM_OK) return s;
    if ((s = ensure_query_capacity(b->m, nq, st)) != PM_OK) return s;
    if ((s = batch_upload_queries(b, descs, query_offsets, &kmax, &nbr_total)) != PM_OK) return s;
    return batch_query_device(b, kmax, d_qpos4, d_qnrm4, nq, d_rad4, d_nbr, d_r2, d_count, st);
}

pm_status pm_batch_capture(pm_batch* b, const float* d_pos4, const float* d_pow4, const uint32_t* photon_offsets,
                           uint32_t num_maps, int format, const pm_query_desc* descs, const float* d_qpos4,
                           const float* d_qnrm4, const uint32_t* query_offsets, float* d_rad4, uint32_t* d_nbr,
                           float* d_r2, uint32_t* d_count) {
    if (!b) return PM_ERR_INVALID;
    pm_status s = batch_prepare_build(b, d_pos4, d_pow4, photon_offsets, num_maps, format);
    if (s != PM_OK) return s;
    b->built = true;   // the tables describe the maps the graph will build
    uint32_t nq = 0, kmax = 1;
    uint64_t nbr_total = 0;
    if ((s = batch_check_query_args(b, query_offsets, d_qpos4, d_qnrm4, d_rad4, &nq)) != PM_OK) return s;
    if ((s = ensure_query_capacity(b->m, nq, nullptr)) != PM_OK) return s;
    if ((s = batch_upload_queries(b, descs, query_offsets, &kmax, &nbr_total)) != PM_OK) return s;
    if (!b->cap_stream && cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
        return check_cuda(b->m, "pm_batch_capture: stream");
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    // kernel attributes are set outside the capture
    if (cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return check_cuda(b->m, "pm_batch_capture: begin");
    pm_status sb = batch_build_device(b, d_pos4, d_pow4, format, b->cap_stream);
    pm_status sq = sb == PM_OK ? batch_query_device(b, kmax, d_qpos4, d_qnrm4, nq, d_rad4, d_nbr, d_r2, d_count,
                                                    b->cap_stream)
                               : sb;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    if (sq != PM_OK) { if (g) cudaGraphDestroy(g); return sq; }
    if (e != cudaSuccess || !g) return check_cuda(b->m, "pm_batch_capture: end");
    b->graph = g;
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) return check_cuda(b->m, "pm_batch_capture: instantiate");
    b->m->n = b->total_photons;
    b->m->built = true;
    return PM_OK;
}

pm_status pm_batch_launch(pm_batch* b, void* stream) {
    if (!b) return PM_ERR_INVALID;
    if (!b->exec) return batch_fail(b, PM_ERR_STATE, "no captured batch; call pm_batch_capture first");
    if (cudaGraphLaunch(b->exec, reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
        return check_cuda(b->m, "pm_batch_launch");
    return PM_OK;
}

pm_status pm_batch_get_info(pm_batch* b, pm_map_info* info, void* stream) {
    if (!b) return PM_ERR_INVALID;
    return pm_get_info(b->m, info, stream);
}

const char* pm_batch_last_error(const pm_batch* b) { return b ? pm_last_error(b->m) : "null handle"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner: times build + query for a grid of tuning candidates on a strided
// sample of the caller's queries and keeps the fastest (build time plus query
// time scaled to all queries).  Leaf size changes the build, so every
// candidate rebuilds the map.
namespace {

struct TuneCand {
    uint32_t leaf;
    int wpb, rounds, qpw, layout;
};

std::vector<TuneCand> tune_candidates(uint32_t k) {
    std::vector<TuneCand> c;
    const uint32_t leaves[] = {16, 24, 32, 48, 64};
    const int wpbs[] = {2, 4, 8};
    const int rounds[] = {8, 32};
    for (uint32_t l : leaves)
        for (int w : wpbs)
            for (int r : rounds) {
                c.push_back({l, w, r, 1, PM_KBUF_GROUP});
                c.push_back({l, w, r, 2, PM_KBUF_GROUP});
                c.push_back({l, w, r, 1, PM_KBUF_WIDE});
            }
    if (k <= 64) c.push_back({16, 4, 8, 1, PM_KBUF_HEAP});   // one lane per query suits small k
    return c;
}

}  // namespace

extern "C" pm_status pm_autotune(pm_map* m, const float* d_pos4, const float* d_pow4, uint32_t n, int format,
                                 const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4, uint32_t nq,
                                 uint32_t max_sample, pm_tuning* best, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (!best) return fail(m, PM_ERR_INVALID, "best is NULL");
    pm_status s = validate_desc(m, desc, true);
    if (s != PM_OK) return s;
    if (nq == 0 || n == 0) return fail(m, PM_ERR_INVALID, "autotuning needs photons and queries");
    if (!d_qpos4 || !d_qnrm4 || !aligned16(d_qpos4) || !aligned16(d_qnrm4))
        return fail(m, PM_ERR_INVALID, "query arrays must be non-NULL and 16-byte aligned");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (capturing(st)) return fail(m, PM_ERR_STATE, "pm_autotune cannot run inside a stream capture");
    const uint32_t sample = max_sample == 0 || max_sample > nq ? nq : max_sample;
    const uint32_t stride = nq / sample;
    if ((s = ensure_query_capacity(m, sample, st)) != PM_OK) return s;
    if ((s = buf_ensure(m, m->gnrm, (size_t)sample * sizeof(float4), "tune normals")) != PM_OK) return s;
    if ((s = buf_ensure(m, m->gest, (size_t)sample * sizeof(float4), "tune estimates")) != PM_OK) return s;
    DevBuf spos;
    if ((s = buf_ensure(m, spos, (size_t)sample * sizeof(float4), "tune positions")) != PM_OK) return s;
    // strided sample: every stride-th query (one 16-byte record per row)
    if (cudaMemcpy2DAsync(spos.ptr, sizeof(float4), d_qpos4, (size_t)stride * sizeof(float4), sizeof(float4), sample,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpy2DAsync(m->gnrm.ptr, sizeof(float4), d_qnrm4, (size_t)stride * sizeof(float4), sizeof(float4), sample,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        buf_free(m, spos);
        return check_cuda(m, "pm_autotune: sample");
    }
    cudaEvent_t ev[3];
    for (cudaEvent_t& e : ev) cudaEventCreate(&e);
    const uint32_t saved_leaf = m->leaf_size;
    const int saved[4] = {m->warps_per_block, m->rounds_per_chunk, m->queries_per_warp, m->kbuf_layout};
    float best_score = INFINITY;
    TuneCand best_c{saved_leaf, saved[0], saved[1], saved[2], saved[3]};
    float best_b = 0, best_q = 0;
    const double scale = (double)nq / (double)sample;
    for (const TuneCand& c : tune_candidates(desc->k)) {
        m->leaf_size = c.leaf; m->warps_per_block = c.wpb; m->rounds_per_chunk = c.rounds;
        m->queries_per_warp = c.qpw; m->kbuf_layout = c.layout;
        float tb = 0, tq = 0;
        for (int rep = 0; rep < 2; ++rep) {   // the second run is timed
            cudaEventRecord(ev[0], st);
            s = pm_build(m, d_pos4, d_pow4, n, format, stream);
            cudaEventRecord(ev[1], st);
            if (s == PM_OK)
                s = pm_query(m, desc, static_cast<const float*>(spos.ptr), static_cast<const float*>(m->gnrm.ptr), sample,
                             static_cast<float*>(m->gest.ptr), nullptr, nullptr, nullptr, stream);
            cudaEventRecord(ev[2], st);
            if (s != PM_OK) break;
            cudaEventSynchronize(ev[2]);
            cudaEventElapsedTime(&tb, ev[0], ev[1]);
            cudaEventElapsedTime(&tq, ev[1], ev[2]);
        }
        if (s != PM_OK) break;
        const float score = tb + (float)(tq * scale);
        if (score < best_score) { best_score = score; best_c = c; best_b = tb; best_q = (float)(tq * scale); }
    }
    for (cudaEvent_t& e : ev) cudaEventDestroy(e);
    buf_free(m, spos);
    if (s != PM_OK) {
        m->leaf_size = saved_leaf; m->warps_per_block = saved[0]; m->rounds_per_chunk = saved[1];
        m->queries_per_warp = saved[2]; m->kbuf_layout = saved[3];
        return s;
    }
    m->leaf_size = best_c.leaf; m->warps_per_block = best_c.wpb; m->rounds_per_chunk = best_c.rounds;
    m->queries_per_warp = best_c.qpw; m->kbuf_layout = best_c.layout;
    best->leaf_size = best_c.leaf; best->warps_per_block = best_c.wpb; best->rounds_per_chunk = best_c.rounds;
    best->queries_per_warp = best_c.qpw; best->kbuf_layout = best_c.layout;
    best->build_ms = best_b; best->query_ms = best_q;
    // leave the map built with the chosen leaf size
    return pm_build(m, d_pos4, d_pow4, n, format, stream);
}

extern "C" pm_status pm_batch_autotune(pm_batch* b, const float* d_pos4, const float* d_pow4,
                                       const uint32_t* photon_offsets, uint32_t num_maps, int format,
                                       const pm_query_desc* descs, const float* d_qpos4, const float* d_qnrm4,
                                       const uint32_t* query_offsets, float* d_rad4, pm_tuning* best, void* stream) {
    if (!b) return PM_ERR_INVALID;
    if (!best) return batch_fail(b, PM_ERR_INVALID, "best is NULL");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (capturing(st)) return batch_fail(b, PM_ERR_STATE, "pm_batch_autotune cannot run inside a stream capture");
    pm_map* m = b->m;
    cudaEvent_t ev[3];
    for (cudaEvent_t& e : ev) cudaEventCreate(&e);
    const uint32_t saved_leaf = m->leaf_size;
    const int saved_wpb = m->warps_per_block, saved_rounds = m->rounds_per_chunk;
    float best_score = INFINITY, best_b = 0, best_q = 0;
    uint32_t bl = saved_leaf;
    int bw = saved_wpb, br = saved_rounds;
    pm_status s = PM_OK;
    const uint32_t leaves[] = {16, 24, 32, 48, 64};
    const int wpbs[] = {2, 4, 8};
    const int rounds[] = {8, 32};
    const int layouts[] = {PM_KBUF_GROUP, PM_KBUF_WIDE};
    int blay = PM_KBUF_WIDE;
    for (uint32_t l : leaves)
        for (int w : wpbs)
            for (int r : rounds)
              for (int lay : layouts) {
                m->leaf_size = l; m->warps_per_block = w; m->rounds_per_chunk = r;
                m->queries_per_warp = 1; m->kbuf_layout = lay;
                float tb = 0, tq = 0;
                for (int rep = 0; rep < 2 && s == PM_OK; ++rep) {
                    cudaEventRecord(ev[0], st);
                    s = pm_batch_build(b, d_pos4, d_pow4, photon_offsets, num_maps, format, stream);
                    cudaEventRecord(ev[1], st);
                    if (s == PM_OK)
                        s = pm_batch_query(b, descs, d_qpos4, d_qnrm4, query_offsets, d_rad4, nullptr, nullptr, nullptr,
                                           stream);
                    cudaEventRecord(ev[2], st);
                    cudaEventSynchronize(ev[2]);
                    cudaEventElapsedTime(&tb, ev[0], ev[1]);
                    cudaEventElapsedTime(&tq, ev[1], ev[2]);
                }
                if (s != PM_OK) break;
                if (tb + tq < best_score) {
                    best_score = tb + tq; bl = l; bw = w; br = r; blay = lay; best_b = tb; best_q = tq;
                }
              }
    for (cudaEvent_t& e : ev) cudaEventDestroy(e);
    m->leaf_size = s == PM_OK ? bl : saved_leaf;
    m->warps_per_block = s == PM_OK ? bw : saved_wpb;
    m->rounds_per_chunk = s == PM_OK ? br : saved_rounds;
    m->queries_per_warp = 1;
    m->kbuf_layout = s == PM_OK ? blay : PM_KBUF_GROUP;
    if (s != PM_OK) return s;
    best->leaf_size = bl; best->warps_per_block = bw; best->rounds_per_chunk = br;
    best->queries_per_warp = 1; best->kbuf_layout = blay;
    best->build_ms = best_b; best->query_ms = best_q;
    return pm_batch_build(b, d_pos4, d_pow4, photon_offsets, num_maps, format, stream);
}

// ---------------------------------------------------------------------------
// Photon ingest: PhotonMap::Merge (PhotonMap.cpp:181-184) over
// PhotonData::Merge (KernelDefs.cpp:363-384).
extern "C" pm_status pm_merge(pm_map* m, const float* d_pos4, const float* d_pow4, const uint32_t* d_is_valid,
                              uint32_t n, uint32_t* merged, void* stream) {
    if (!m) return PM_ERR_INVALID;
    if (merged) *merged = 0;
    if (n == 0) return PM_OK;
    if (!d_pos4 || !d_pow4) return fail(m, PM_ERR_INVALID, "photon arrays must be non-NULL");
    if (!aligned16(d_pos4) || !aligned16(d_pow4)) return fail(m, PM_ERR_INVALID, "photon arrays must be 16-byte aligned");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (capturing(st)) return fail(m, PM_ERR_STATE, "pm_merge is synchronous and cannot be captured");
    pm_status s;
    if ((s = buf_ensure(m, m->mflags, (size_t)n * sizeof(uint32_t), "merge flags")) != PM_OK) return s;
    if ((s = buf_ensure(m, m->mrank, (size_t)n * sizeof(uint32_t), "merge ranks")) != PM_OK) return s;
    if ((s = buf_ensure(m, m->mscan, (scan_scratch_words(n) + 1) * sizeof(uint32_t), "merge scan")) != PM_OK) return s;
    uint32_t* total = P<uint32_t>(m->mscan);
    int nl = merge_ranks(d_is_valid, n, P<uint32_t>(m->mflags), P<uint32_t>(m->mrank), total + 1, total, st);
    uint32_t count = 0;
    if (cudaMemcpyAsync(&count, total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return check_cuda(m, "pm_merge");
    const uint64_t need = (uint64_t)m->merged_n + count;
    if (m->max_photons && need > m->max_photons)
        return fail(m, PM_ERR_INVALID, "merging %u photons exceeds the map's max_photons = %u", count, m->max_photons);
    if (need > 0x7fffffffull) return fail(m, PM_ERR_UNSUPPORTED, "more than 2^31 - 1 photons");
    if (need > m->cap_merged) {   // grow, keeping what is merged already
        const uint32_t cap = (uint32_t)std::max<uint64_t>(need, m->max_photons ? m->max_photons : need);
        DevBuf np, nw;
        if ((s = buf_ensure(m, np, (size_t)cap * sizeof(float4), "merged positions")) != PM_OK) return s;
        if ((s = buf_ensure(m, nw, (size_t)cap * sizeof(float4), "merged powers")) != PM_OK) { buf_free(m, np); return s; }
        if (m->merged_n) {
            cudaMemcpyAsync(np.ptr, m->mpos.ptr, (size_t)m->merged_n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(nw.ptr, m->mpow.ptr, (size_t)m->merged_n * sizeof(float4), cudaMemcpyDeviceToDevice, st);
            cudaStreamSynchronize(st);
        }
        buf_free(m, m->mpos);
        buf_free(m, m->mpow);
        m->mpos = np;
        m->mpow = nw;
        m->cap_merged = cap;
    }
    if (count) {
        nl += merge_scatter(reinterpret_cast<const float4*>(d_pos4), reinterpret_cast<const float4*>(d_pow4),
                            P<uint32_t>(m->mflags), P<uint32_t>(m->mrank), n, P<float4>(m->mpos) + m->merged_n,
                            P<float4>(m->mpow) + m->merged_n, st);
    }
    m->merged_n += count;
    m->launches += (uint64_t)nl;
    if (merged) *merged = count;
    return check_cuda(m, "pm_merge");
}

extern "C" pm_status pm_build_merged(pm_map* m, int format, void* stream) {
    if (!m) return PM_ERR_INVALID;
    return pm_build(m, m->merged_n ? static_cast<const float*>(m->mpos.ptr) : nullptr,
                    m->merged_n ? static_cast<const float*>(m->mpow.ptr) : nullptr, m->merged_n, format, stream);
}

extern "C" pm_status pm_clear_merged(pm_map* m) {
    if (!m) return PM_ERR_INVALID;
    m->merged_n = 0;
    return PM_OK;
}

extern "C" pm_status pm_merged_count(const pm_map* m, uint32_t* count) {
    if (!m || !count) return PM_ERR_INVALID;
    *count = m->merged_n;
    return PM_OK;
}
