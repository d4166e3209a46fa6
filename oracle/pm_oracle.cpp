// pm_oracle.cpp -- CPU oracle for the photon-map kNN radiance estimate.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
// mnrt_b200/; it is linked only by tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py.  The product never calls it.
//
// PARITY UNPINNED: the reference (jonike/mnrt) ships no tests, golden vectors
// or fixtures for this path, and its path cannot be compiled here (legacy
// texture<> references removed in CUDA 12, the absent CUDA-SDK cutil headers
// and the absent, unvendored CUDPP library).  The oracle therefore restates
// the reference's algorithm from its source and is cross-checked against an
// independent numpy restatement and the committed fixtures in tests/golden/.
//
// What is restated, and from where (paths inside the reference project):
//   * range membership is strict:  d^2 < r^2                GPU/photon_knn.cu:189
//   * front-face test: dot(n, -inDir) > 0 -> weight 1 else 0 GPU/photon_knn.cu:196-208
//   * estimate E = sum(alpha * flux) / (pi * r^2_used), with
//     r^2_used = max d^2 of the found photons when >= k were found,
//     otherwise the query radius^2; E = 0 when r^2_used == 0  GPU/photon_knn.cu:221-232
//   * estimates from fewer than 8 photons are zeroed          GPU/photon_knn.cu:518-519
//     (exposed as the min_found parameter)
//   * photon layout: position.w = azimuth phi, power.w = polar theta,
//     direction = (sin t cos p, sin t sin p, cos t)           GPU/photon_dev.h:71-113,
//                                                              GPU/mncudautil_dev.h:345-352
//
// The engine's own contract on top of that (it defines "exact kNN", which the
// reference only approximates, Help/MNRT_Documentation.html section 4.2):
//   * d^2 = ((dx*dx) + (dy*dy)) + (dz*dz), dx = px - qx, every operation
//     rounded to nearest FP32 with no contraction (build with -ffp-contract=off)
//   * N(q) = the k photons with the smallest (d^2, photon index) among those
//     with d^2 < R^2;  count = |N(q)|;  r^2 = d^2 of the k-th when count == k,
//     else R^2 (R^2 itself rounded in FP32)
//   * incident directions are stored octahedral-encoded in 2 x 16 bits; the
//     front test runs in FP32 on the decoded (unnormalised) vector
//   * cone filter (Jensen 2001): w = 1 - d/(kc r), norm 1/((1 - 2/(3kc)) pi r^2)
//     Epanechnikov (2-D):        w = 1 - d^2/r^2, norm 2/(pi r^2)
//     box (the reference's):     w = 1,           norm 1/(pi r^2)
//
// Build: see oracle/Makefile (g++ -O2 -ffp-contract=off -fno-fast-math).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#ifdef __FAST_MATH__
#error "the oracle must be built without -ffast-math (IEEE rounding of every operation)"
#endif
// x86-64 evaluates float/double in SSE registers (FLT_EVAL_METHOD == 0) and
// -ffp-contract=off keeps every a*b+c as two roundings.

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// ---------------------------------------------------------------- contract --

// Squared distance, fixed evaluation order, FP32, no contraction.
inline float d2_f32(float qx, float qy, float qz, float px, float py, float pz) {
    float dx = px - qx, dy = py - qy, dz = pz - qz;
    float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    float s = xx + yy;
    return s + zz;
}

// Octahedral direction code: 16-bit snorm u (low half) and v (high half).
inline void oct_decode(uint32_t bits, float out[3]) {
    int16_t iu = (int16_t)(bits & 0xffffu), iv = (int16_t)(bits >> 16);
    const float s = 1.0f / 32767.0f;
    float fu = (float)iu * s, fv = (float)iv * s;
    float au = std::fabs(fu), av = std::fabs(fv);
    float z = (1.0f - au) - av;
    float x = fu, y = fv;
    if (z < 0.0f) {
        x = (1.0f - av) * (fu >= 0.0f ? 1.0f : -1.0f);
        y = (1.0f - au) * (fv >= 0.0f ? 1.0f : -1.0f);
    }
    out[0] = x; out[1] = y; out[2] = z;
}

inline int32_t snorm16(float f) {
    float t = f * 32767.0f;
    float r = std::nearbyint(t);  // round half to even (default rounding mode)
    if (r > 32767.0f) r = 32767.0f;
    if (r < -32767.0f) r = -32767.0f;
    return (int32_t)r;
}

inline uint32_t oct_encode(float dx, float dy, float dz) {
    float s = (std::fabs(dx) + std::fabs(dy)) + std::fabs(dz);
    if (!(s > 0.0f)) return 0u;  // degenerate direction -> (0,0,1)
    float px = dx / s, py = dy / s;
    if (dz < 0.0f) {
        float ax = std::fabs(px), ay = std::fabs(py);
        float nx = (1.0f - ay) * (px >= 0.0f ? 1.0f : -1.0f);
        float ny = (1.0f - ax) * (py >= 0.0f ? 1.0f : -1.0f);
        px = nx; py = ny;
    }
    uint32_t u = (uint32_t)(snorm16(px) & 0xffff), v = (uint32_t)(snorm16(py) & 0xffff);
    return u | (v << 16);
}

// front: dot(n, -dir) > 0, FP32, fixed order.
inline bool front_f32(float nx, float ny, float nz, uint32_t dirbits) {
    float d[3];
    oct_decode(dirbits, d);
    float a = nx * (-d[0]), b = ny * (-d[1]), c = nz * (-d[2]);
    float s = a + b;
    return (s + c) > 0.0f;
}

// Deterministic sin/cos in FP64 for the spherical ingest: Cody-Waite
// reduction by pi/2 (split into a 33-bit head and a tail) and Taylor series
// to degree 21/22 on [-pi/4, pi/4].  Every operation is a single IEEE double
// rounding, so the CUDA side (explicit __dmul_rn/__dadd_rn) gives the same bits.
constexpr double kPio2Hi = 0x1.921fb544p+0;            // pi/2 to 33 bits
constexpr double kPio2Lo = 0x1.0b4611a626331p-34;      // pi/2 - kPio2Hi
constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;    // 2/pi

inline void sincos_det(double x, double* s_out, double* c_out) {
    double kq = std::nearbyint(x * kTwoOverPi);
    double t1 = kq * kPio2Hi;
    double r0 = x - t1;
    double t2 = kq * kPio2Lo;
    double r = r0 - t2;
    double r2 = r * r;
    // sin(r) = r * (1 - r2/3! + r2^2/5! - ...), Horner over r2
    double ps = 1.0 / 51090942171709440000.0;  // 1/21!
    const double sc[] = {1.0 / 121645100408832000.0, 1.0 / 355687428096000.0,
                         1.0 / 1307674368000.0, 1.0 / 6227020800.0, 1.0 / 39916800.0,
                         1.0 / 362880.0, 1.0 / 5040.0, 1.0 / 120.0, 1.0 / 6.0, 1.0};
    const double sg[] = {-1.0, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0};
    // coefficient of r^(2j+1) is (-1)^j / (2j+1)!; j = 10 .. 0
    ps = ps;  // (-1)^10 = +1
    for (int i = 0; i < 10; ++i) {
        double m = ps * r2;
        ps = m + sg[i] * sc[i];
    }
    double sv = ps * r;
    // cos(r) = 1 - r2/2! + ..., coefficient of r^(2j) is (-1)^j/(2j)!; j = 11 .. 0
    double pc = -1.0 / 1124000727777607680000.0;  // -1/22!
    const double cc[] = {1.0 / 2432902008176640000.0, 1.0 / 6402373705728000.0,
                         1.0 / 20922789888000.0, 1.0 / 87178291200.0, 1.0 / 479001600.0,
                         1.0 / 3628800.0, 1.0 / 40320.0, 1.0 / 720.0, 1.0 / 24.0, 1.0 / 2.0, 1.0};
    const double cg[] = {1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0};
    for (int i = 0; i < 11; ++i) {
        double m = pc * r2;
        pc = m + cg[i] * cc[i];
    }
    double cv = pc;
    long q = ((long)kq) & 3;
    double s, c;
    switch (q) {
        case 0: s = sv; c = cv; break;
        case 1: s = cv; c = -sv; break;
        case 2: s = -sv; c = -cv; break;
        default: s = -cv; c = sv; break;
    }
    *s_out = s; *c_out = c;
}

inline uint32_t spherical_to_oct(float phi, float theta) {
    double sp, cp, st, ct;
    sincos_det((double)phi, &sp, &cp);
    sincos_det((double)theta, &st, &ct);
    double x = st * cp, y = st * sp;
    return oct_encode((float)x, (float)y, (float)ct);
}

inline uint64_t key_of(float d2, uint32_t idx) { return ((uint64_t)f2u(d2) << 32) | idx; }

template <class F>
void parallel_for_blocks(int64_t n, int64_t block, int nthreads, F&& f) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (n <= 0) return;
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(block);
            if (b >= n) break;
            f(b, std::min(n, b + block));
        }
    };
    if (nthreads == 1) { worker(); return; }
    std::vector<std::thread> th;
    th.reserve(nthreads);
    for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
}

// Bounded max-heap of (d2, idx) keys, size <= k.
struct KHeap {
    uint64_t* a; uint32_t n; uint32_t k;
    void push(uint64_t v) {
        if (n < k) {
            uint32_t i = n++;
            while (i > 0) { uint32_t p = (i - 1) >> 1; if (a[p] >= v) break; a[i] = a[p]; i = p; }
            a[i] = v;
        } else if (v < a[0]) {
            uint32_t i = 0;
            for (;;) {
                uint32_t l = 2 * i + 1; if (l >= n) break;
                uint32_t c = (l + 1 < n && a[l + 1] > a[l]) ? l + 1 : l;
                if (a[c] <= v) break;
                a[i] = a[c]; i = c;
            }
            a[i] = v;
        }
    }
    bool full() const { return n == k; }
    uint64_t top() const { return a[0]; }
};

inline void finish_query(KHeap& h, float R2, uint32_t k, uint32_t* out_idx, float* out_d2,
                         uint32_t* out_count, float* out_r2) {
    std::sort(h.a, h.a + h.n);
    for (uint32_t j = 0; j < k; ++j) {
        if (j < h.n) { out_idx[j] = (uint32_t)(h.a[j] & 0xffffffffu); out_d2[j] = u2f((uint32_t)(h.a[j] >> 32)); }
        else { out_idx[j] = 0xffffffffu; out_d2[j] = INFINITY; }
    }
    *out_count = h.n;
    *out_r2 = (h.n == k) ? u2f((uint32_t)(h.a[k - 1] >> 32)) : R2;
}

// ------------------------------------------------------ CPU point kd-tree --
// Median split on the longest axis of the node's point bounds (the
// reference's large-node rule, GPU/kdtree.cu:629-682, without its
// empty-space cuts), leaves of <= kLeaf points.
constexpr int kLeaf = 12;

struct KdNode { float split; int32_t axis; int32_t left, right; int32_t begin, end; };

struct KdTree {
    std::vector<float> x, y, z;    // points in tree order
    std::vector<uint32_t> idx;     // original photon index
    std::vector<KdNode> nodes;
    uint32_t n = 0;
};

int kd_build_rec(KdTree& t, std::vector<uint32_t>& ord, const float* pos4, int b, int e) {
    int me = (int)t.nodes.size();
    t.nodes.push_back(KdNode{0.f, -1, -1, -1, b, e});
    if (e - b <= kLeaf) return me;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = b; i < e; ++i)
        for (int a = 0; a < 3; ++a) { float v = pos4[4 * (size_t)ord[i] + a]; lo[a] = std::min(lo[a], v); hi[a] = std::max(hi[a], v); }
    int axis = 0;
    for (int a = 1; a < 3; ++a) if (hi[a] - lo[a] > hi[axis] - lo[axis]) axis = a;
    int mid = b + (e - b) / 2;
    std::nth_element(ord.begin() + b, ord.begin() + mid, ord.begin() + e, [&](uint32_t u, uint32_t v) {
        float fu = pos4[4 * (size_t)u + axis], fv = pos4[4 * (size_t)v + axis];
        return fu < fv || (fu == fv && u < v);
    });
    float split = pos4[4 * (size_t)ord[mid] + axis];
    int l = kd_build_rec(t, ord, pos4, b, mid);
    int r = kd_build_rec(t, ord, pos4, mid, e);
    t.nodes[me].split = split; t.nodes[me].axis = axis; t.nodes[me].left = l; t.nodes[me].right = r;
    return me;
}

// The same tree built with the two halves of every split of the top `depth`
// levels on their own threads: each half is a disjoint range of ord, so the
// splits, and with them the points' tree order, are those of kd_build_rec;
// only the node numbering differs (each half's nodes follow its parent's).
// Returns the subtree's nodes with the subtree root first, child links local.
std::vector<KdNode> kd_build_par(std::vector<uint32_t>& ord, const float* pos4, int b, int e, int depth) {
    std::vector<KdNode> out;
    if (depth <= 0 || e - b <= kLeaf) {
        KdTree sub;
        kd_build_rec(sub, ord, pos4, b, e);
        return std::move(sub.nodes);
    }
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = b; i < e; ++i)
        for (int a = 0; a < 3; ++a) { float v = pos4[4 * (size_t)ord[i] + a]; lo[a] = std::min(lo[a], v); hi[a] = std::max(hi[a], v); }
    int axis = 0;
    for (int a = 1; a < 3; ++a) if (hi[a] - lo[a] > hi[axis] - lo[axis]) axis = a;
    const int mid = b + (e - b) / 2;
    std::nth_element(ord.begin() + b, ord.begin() + mid, ord.begin() + e, [&](uint32_t u, uint32_t v) {
        float fu = pos4[4 * (size_t)u + axis], fv = pos4[4 * (size_t)v + axis];
        return fu < fv || (fu == fv && u < v);
    });
    const float split = pos4[4 * (size_t)ord[mid] + axis];   // before the halves reorder their ranges
    std::vector<KdNode> left, right;
    std::thread th([&] { left = kd_build_par(ord, pos4, b, mid, depth - 1); });
    right = kd_build_par(ord, pos4, mid, e, depth - 1);
    th.join();
    out.reserve(1 + left.size() + right.size());
    out.push_back(KdNode{split, axis, 1, (int32_t)(1 + left.size()), b, e});
    auto append = [&](const std::vector<KdNode>& sub, int32_t off) {
        for (KdNode nd : sub) {
            if (nd.axis >= 0) { nd.left += off; nd.right += off; }
            out.push_back(nd);
        }
    };
    append(left, 1);
    append(right, (int32_t)(1 + left.size()));
    return out;
}

void kd_query(const KdTree& t, float qx, float qy, float qz, float R2, KHeap& h) {
    struct Ent { int32_t node; float lb; };
    Ent stack[128];
    int sp = 0;
    stack[sp++] = Ent{0, 0.0f};
    const float q[3] = {qx, qy, qz};
    while (sp > 0) {
        Ent e = stack[--sp];
        if (e.lb >= R2) continue;
        if (h.full() && e.lb > u2f((uint32_t)(h.top() >> 32))) continue;
        const KdNode* nd = &t.nodes[e.node];
        while (nd->axis >= 0) {
            // plane lower bound: |p_a - q_a| >= |split - q_a| for the far side
            float diff = nd->split - q[nd->axis];
            float lbp = diff * diff;
            int nearc, farc;
            if (q[nd->axis] < nd->split) { nearc = nd->left; farc = nd->right; }
            else { nearc = nd->right; farc = nd->left; }
            float flb = std::max(e.lb, lbp);
            if (flb < R2 && sp < 128) stack[sp++] = Ent{farc, flb};
            nd = &t.nodes[nearc];
        }
        for (int i = nd->begin; i < nd->end; ++i) {
            float d2 = d2_f32(qx, qy, qz, t.x[i], t.y[i], t.z[i]);
            if (d2 < R2) h.push(key_of(d2, t.idx[i]));
        }
    }
}

}  // namespace

extern "C" {

int orc_version(void) { return 3; }

float orc_d2(float qx, float qy, float qz, float px, float py, float pz) { return d2_f32(qx, qy, qz, px, py, pz); }
uint32_t orc_oct_encode(float x, float y, float z) { return oct_encode(x, y, z); }
void orc_oct_decode(uint32_t bits, float* out3) { oct_decode(bits, out3); }
int orc_front(float nx, float ny, float nz, uint32_t dirbits) { return front_f32(nx, ny, nz, dirbits) ? 1 : 0; }
void orc_sincos(double x, double* sc) { sincos_det(x, &sc[0], &sc[1]); }
uint32_t orc_spherical_to_oct(float phi, float theta) { return spherical_to_oct(phi, theta); }

// Convert reference-format photons (pos.w = azimuth, pow.w = polar angle) to
// the engine's packed record (pos.w = photon index bits, pow.w = oct bits).
void orc_pack_reference_photons(const float* pos4, const float* pow4, uint32_t n, float* out_pos4, float* out_pow4) {
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t dir = spherical_to_oct(pos4[4 * (size_t)i + 3], pow4[4 * (size_t)i + 3]);
        for (int a = 0; a < 3; ++a) { out_pos4[4 * (size_t)i + a] = pos4[4 * (size_t)i + a]; out_pow4[4 * (size_t)i + a] = pow4[4 * (size_t)i + a]; }
        out_pos4[4 * (size_t)i + 3] = u2f(i);
        out_pow4[4 * (size_t)i + 3] = u2f(dir);
    }
}

// Exact kNN by brute force (the definition itself).  pos4: photons in caller
// order (index = position in the array); q4: query positions.
void orc_knn_brute(const float* pos4, uint32_t n, const float* q4, uint32_t nq, uint32_t k, float R,
                   uint32_t* out_idx, float* out_d2, uint32_t* out_count, float* out_r2, int nthreads) {
    const float R2 = R * R;
    parallel_for_blocks(nq, 64, nthreads, [&](int64_t b, int64_t e) {
        std::vector<uint64_t> buf(k ? k : 1);
        for (int64_t q = b; q < e; ++q) {
            KHeap h{buf.data(), 0, k};
            float qx = q4[4 * q], qy = q4[4 * q + 1], qz = q4[4 * q + 2];
            if (k > 0)
                for (uint32_t i = 0; i < n; ++i) {
                    float d2 = d2_f32(qx, qy, qz, pos4[4 * (size_t)i], pos4[4 * (size_t)i + 1], pos4[4 * (size_t)i + 2]);
                    if (d2 < R2) h.push(key_of(d2, i));
                }
            finish_query(h, R2, k, out_idx + (size_t)q * k, out_d2 + (size_t)q * k, out_count + q, out_r2 + q);
        }
    });
}

// CPU baseline: median-split point kd-tree + bounded-heap kNN, multithreaded
// over query blocks.  Same results as orc_knn_brute (tree-independent).
void* orc_kdtree_build(const float* pos4, uint32_t n) {
    KdTree* t = new KdTree();
    t->n = n;
    std::vector<uint32_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0u);
    t->nodes.reserve(2 * (n / kLeaf + 1) + 1);
    if (n > 0) kd_build_rec(*t, ord, pos4, 0, (int)n);
    else t->nodes.push_back(KdNode{0.f, -1, -1, -1, 0, 0});
    t->x.resize(n); t->y.resize(n); t->z.resize(n); t->idx.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        t->x[i] = pos4[4 * (size_t)ord[i]]; t->y[i] = pos4[4 * (size_t)ord[i] + 1]; t->z[i] = pos4[4 * (size_t)ord[i] + 2];
        t->idx[i] = ord[i];
    }
    return t;
}

// Multithreaded build (the top levels' halves on their own threads, up to
// nthreads in flight; 0 = one per hardware thread): the same splits and tree
// order of the points as orc_kdtree_build.
void* orc_kdtree_build_mt(const float* pos4, uint32_t n, int nthreads) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    int depth = 0;
    while ((1 << depth) < nthreads && depth < 16) ++depth;
    KdTree* t = new KdTree();
    t->n = n;
    std::vector<uint32_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0u);
    if (n > 0) t->nodes = kd_build_par(ord, pos4, 0, (int)n, depth);
    else t->nodes.push_back(KdNode{0.f, -1, -1, -1, 0, 0});
    t->x.resize(n); t->y.resize(n); t->z.resize(n); t->idx.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        t->x[i] = pos4[4 * (size_t)ord[i]]; t->y[i] = pos4[4 * (size_t)ord[i] + 1]; t->z[i] = pos4[4 * (size_t)ord[i] + 2];
        t->idx[i] = ord[i];
    }
    return t;
}

// The points in tree order (caller indices), for tests.
void orc_kdtree_order(const void* h, uint32_t* out) {
    const KdTree& t = *(const KdTree*)h;
    std::copy(t.idx.begin(), t.idx.end(), out);
}

void orc_kdtree_free(void* h) { delete (KdTree*)h; }

void orc_knn_kdtree(const void* tree, const float* q4, uint32_t nq, uint32_t k, float R, uint32_t* out_idx,
                    float* out_d2, uint32_t* out_count, float* out_r2, int nthreads) {
    const KdTree& t = *(const KdTree*)tree;
    const float R2 = R * R;
    parallel_for_blocks(nq, 64, nthreads, [&](int64_t b, int64_t e) {
        std::vector<uint64_t> buf(k ? k : 1);
        for (int64_t q = b; q < e; ++q) {
            KHeap h{buf.data(), 0, k};
            if (k > 0 && t.n > 0) kd_query(t, q4[4 * q], q4[4 * q + 1], q4[4 * q + 2], R2, h);
            finish_query(h, R2, k, out_idx + (size_t)q * k, out_d2 + (size_t)q * k, out_count + q, out_r2 + q);
        }
    });
}

// FP64 radiance over a given neighbour set (the FP32 contract decides the
// set and the front test; weights, sums and the normalisation run in FP64).
// filter: 0 box, 1 cone, 2 Epanechnikov.  out: 3 doubles per query.
void orc_radiance_fp64(const float* pos4, const float* pow4, const float* q4, const float* n4, uint32_t nq,
                       const uint32_t* nbr, const uint32_t* count, uint32_t k, float R, int filter, float cone_k,
                       uint32_t min_found, double* out, int nthreads) {
    parallel_for_blocks(nq, 256, nthreads, [&](int64_t b, int64_t e) {
        for (int64_t q = b; q < e; ++q) {
            double acc[3] = {0, 0, 0};
            uint32_t cnt = count[q];
            const double qx = q4[4 * q], qy = q4[4 * q + 1], qz = q4[4 * q + 2];
            double r2 = (double)R * (double)R;
            if (cnt == k && k > 0) {
                uint32_t pk = nbr[(size_t)q * k + k - 1];
                double dx = pos4[4 * (size_t)pk] - qx, dy = pos4[4 * (size_t)pk + 1] - qy, dz = pos4[4 * (size_t)pk + 2] - qz;
                r2 = dx * dx + dy * dy + dz * dz;
            }
            if (cnt < min_found || !(r2 > 0.0)) { out[3 * q] = out[3 * q + 1] = out[3 * q + 2] = 0.0; continue; }
            double r = std::sqrt(r2);
            for (uint32_t j = 0; j < cnt; ++j) {
                uint32_t p = nbr[(size_t)q * k + j];
                if (!front_f32(n4[4 * q], n4[4 * q + 1], n4[4 * q + 2], f2u(pow4[4 * (size_t)p + 3]))) continue;
                double dx = pos4[4 * (size_t)p] - qx, dy = pos4[4 * (size_t)p + 1] - qy, dz = pos4[4 * (size_t)p + 2] - qz;
                double d2 = dx * dx + dy * dy + dz * dz;
                double w = 1.0;
                if (filter == 1) w = 1.0 - std::sqrt(d2) / ((double)cone_k * r);
                else if (filter == 2) w = 1.0 - d2 / r2;
                for (int c = 0; c < 3; ++c) acc[c] += w * (double)pow4[4 * (size_t)p + c];
            }
            double norm;
            if (filter == 1) norm = 1.0 / ((1.0 - 2.0 / (3.0 * (double)cone_k)) * kPi * r2);
            else if (filter == 2) norm = 2.0 / (kPi * r2);
            else norm = 1.0 / (kPi * r2);
            for (int c = 0; c < 3; ++c) out[3 * q + c] = acc[c] * norm;
        }
    });
}

// Host reference gradient of a loss L through the FP64 estimate above, for
// given neighbour sets (rows sorted by (d^2, index)).  grad: dL/dE, 3 doubles
// per query.  Writes dL/dpower and dL/dposition, 3 doubles per photon.  The
// adjoint has no reference counterpart; it differentiates E = norm(r^2) *
// sum front * w(d^2, r^2) * flux with r^2 = d^2 of the k-th neighbour (when k
// were found), so the k-th neighbour's position also moves every weight and
// the normalisation of its query.  Single-threaded, queries in order.
void orc_backward_fp64(const float* pos4, const float* pow4, const float* q4, const float* n4, uint32_t n,
                       uint32_t nq, const uint32_t* nbr, const uint32_t* count, uint32_t k, float R, int filter,
                       float cone_k, uint32_t min_found, const double* grad, double* out_gpow, double* out_gpos) {
    std::fill(out_gpow, out_gpow + 3 * (size_t)n, 0.0);
    std::fill(out_gpos, out_gpos + 3 * (size_t)n, 0.0);
    const double kc = (double)cone_k;
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t cnt = count[q];
        const double qx = q4[4 * (size_t)q], qy = q4[4 * (size_t)q + 1], qz = q4[4 * (size_t)q + 2];
        if (!(std::isfinite(qx) && std::isfinite(qy) && std::isfinite(qz))) continue;
        double r2 = (double)R * (double)R;
        const uint32_t* row = nbr + (size_t)q * k;
        if (cnt == k && k > 0) {
            const uint32_t pk = row[k - 1];
            const double dx = pos4[4 * (size_t)pk] - qx, dy = pos4[4 * (size_t)pk + 1] - qy, dz = pos4[4 * (size_t)pk + 2] - qz;
            r2 = dx * dx + dy * dy + dz * dz;
        }
        if (cnt == 0 || cnt < min_found || !(r2 > 0.0)) continue;
        double norm;
        if (filter == 1) norm = 1.0 / ((1.0 - 2.0 / (3.0 * kc)) * kPi * r2);
        else if (filter == 2) norm = 2.0 / (kPi * r2);
        else norm = 1.0 / (kPi * r2);
        const double g[3] = {grad[3 * (size_t)q], grad[3 * (size_t)q + 1], grad[3 * (size_t)q + 2]};
        const double gn[3] = {g[0] * norm, g[1] * norm, g[2] * norm};
        double S[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        for (int pass = 0; pass < 2; ++pass) {
            double Gr = 0.0;
            if (pass == 1 && cnt == k) {
                const double dn = -norm / r2;
                for (int c = 0; c < 3; ++c) Gr += g[c] * (dn * S[c] + norm * T[c]);
            }
            for (uint32_t j = 0; j < cnt; ++j) {
                const uint32_t p = row[j];
                const double dx = pos4[4 * (size_t)p] - qx, dy = pos4[4 * (size_t)p + 1] - qy, dz = pos4[4 * (size_t)p + 2] - qz;
                const double d2 = dx * dx + dy * dy + dz * dz;
                const bool fr = front_f32(n4[4 * (size_t)q], n4[4 * (size_t)q + 1], n4[4 * (size_t)q + 2], f2u(pow4[4 * (size_t)p + 3]));
                double w = 1.0, dwd = 0.0, dwr = 0.0;
                if (filter == 1) {
                    const double d = std::sqrt(d2), r = std::sqrt(r2);
                    w = 1.0 - d / (kc * r);
                    dwd = d > 0.0 ? -1.0 / (2.0 * d * kc * r) : 0.0;
                    dwr = d / (2.0 * kc * r2 * r);
                } else if (filter == 2) {
                    w = 1.0 - d2 / r2;
                    dwd = -1.0 / r2;
                    dwr = d2 / (r2 * r2);
                }
                const double phi[3] = {pow4[4 * (size_t)p], pow4[4 * (size_t)p + 1], pow4[4 * (size_t)p + 2]};
                if (pass == 0) {
                    if (fr)
                        for (int c = 0; c < 3; ++c) { S[c] += w * phi[c]; T[c] += dwr * phi[c]; }
                    continue;
                }
                double coef = 0.0;
                if (fr) {
                    for (int c = 0; c < 3; ++c) out_gpow[3 * (size_t)p + c] += w * gn[c];
                    coef = (gn[0] * phi[0] + gn[1] * phi[1] + gn[2] * phi[2]) * dwd;
                }
                if (j == k - 1) coef += Gr;
                out_gpos[3 * (size_t)p] += 2.0 * coef * dx;
                out_gpos[3 * (size_t)p + 1] += 2.0 * coef * dy;
                out_gpos[3 * (size_t)p + 2] += 2.0 * coef * dz;
            }
        }
    }
}

}  // extern "C"

// ------------------------------------------------------ ZHOU_COMPAT mode --
// The reference's radius pipeline restated on the engine's exported tree
// (nodes: 16 uint32 each = two slots {lo[3], hi[3], ref, cnt}; tree-order
// photons).  Follows KDTreePoint::PrecomputeQueryRadii / ComputeQueryRadii
// (KDTreePoint.cpp:187-248), dev_RefineQueryRadiusZhou / dev_RangeSearchHist
// (GPU/kdtree_point.cu:118-267), kernel_QREEstimateRadii (:453-504) and the
// gather of dev_RangeSearch (GPU/photon_knn.cu:113-235), with the engine's
// stated choices: slots are the tree nodes, the root-to-leaf path follows the
// nearer child box, FP32 steps in a fixed order, histogram index clamped to 31.
namespace {

struct CSlot { float lo[3], hi[3]; uint32_t ref, cnt; };

struct CompatTree {
    const uint32_t* nodes; uint32_t m;   // internal nodes 1..m, node 0 = super-root
    const float* pos; const float* pow;
    CSlot slot(uint32_t sid) const {
        const uint32_t* w = nodes + 16 * (size_t)(sid >> 1) + 8 * (sid & 1u);
        CSlot s;
        for (int a = 0; a < 3; ++a) { s.lo[a] = u2f(w[a]); s.hi[a] = u2f(w[3 + a]); }
        s.ref = w[6]; s.cnt = w[7];
        return s;
    }
};

inline float box_lb_f32(float qx, float qy, float qz, const float* lo, const float* hi) {
    const float q[3] = {qx, qy, qz};
    float g[3];
    for (int a = 0; a < 3; ++a) {
        float x = std::max(lo[a] - q[a], q[a] - hi[a]);
        g[a] = std::max(x, 0.0f);
    }
    float s = g[0] * g[0] + g[1] * g[1];
    return s + g[2] * g[2];
}

template <class F>
void compat_range(const CompatTree& t, float qx, float qy, float qz, float r2, F&& f) {
    std::vector<uint32_t> stack;
    stack.push_back(0u);
    while (!stack.empty()) {
        const uint32_t sid = stack.back();
        stack.pop_back();
        const CSlot s = t.slot(sid);
        if (s.ref == 0xffffffffu) continue;
        if (!(box_lb_f32(qx, qy, qz, s.lo, s.hi) < r2)) continue;
        if (s.cnt > 0) {
            for (uint32_t j = 0; j < s.cnt; ++j) {
                const float* p = t.pos + 4 * (size_t)(s.ref + j);
                const float d2 = d2_f32(qx, qy, qz, p[0], p[1], p[2]);
                if (d2 < r2) f(s.ref + j, d2);
            }
        } else {
            stack.push_back((s.ref << 1) | 1u);
            stack.push_back(s.ref << 1);
        }
    }
}

float compat_refine(const CompatTree& t, float qx, float qy, float qz, float radius_max, uint32_t k, uint32_t iters) {
    float r_min = 0.0f, r_max = radius_max;
    for (uint32_t it = 0; it < iters; ++it) {
        const float r = r_max;
        const float delta = r_max - r_min;
        if (!(delta > 0.0f)) break;
        uint32_t hist[32] = {0};
        compat_range(t, qx, qy, qz, r * r, [&](uint32_t, float d2) {
            const float d = std::sqrt(d2);
            const float fi = (std::max(d - r_min, 0.0f) * 32.0f) / delta;
            uint32_t idx = (uint32_t)fi;
            if (idx > 31) idx = 31;
            if (hist[idx] < 0xfffeu) ++hist[idx];
        });
        uint32_t m = 31, sum = 0;
        for (uint32_t j = 0; j < 32; ++j) {
            sum += hist[j];
            if (sum >= k) { m = j; break; }
        }
        const float inv = 1.0f / 32.0f;
        const float old = r_min;
        r_min = old + ((float)m * delta) * inv;
        r_max = old + ((float)(m + 1) * delta) * inv;
    }
    return r_max;
}

void compat_extent(const CSlot& s, float* c, float& rad) {
    float d2 = 0.0f;
    for (int a = 0; a < 3; ++a) {
        c[a] = (s.lo[a] + s.hi[a]) * 0.5f;
        const float e = s.hi[a] - s.lo[a];
        d2 = a == 0 ? e * e : d2 + e * e;
    }
    rad = std::sqrt(d2) * 0.5f;
}

}  // namespace

extern "C" {

// radius (nq), count (nq), r2_used (nq), rad (3 nq doubles; NULL = radii only)
void orc_compat(const uint32_t* nodes, uint32_t m, const float* tpos4, const float* tpow4, const float* q4,
                const float* n4, uint32_t nq, uint32_t k, float R, uint32_t iters, int filter, float cone_k,
                uint32_t min_found, float* out_radius, uint32_t* out_count, float* out_r2, double* out_rad,
                int nthreads) {
    CompatTree t{nodes, m, tpos4, tpow4};
    const uint32_t nslots = 2 * (m + 1);
    std::vector<float> est(nslots, INFINITY);
    const bool enabled = 2 * m + 1 >= 1000;
    parallel_for_blocks(nslots, 64, nthreads, [&](int64_t b, int64_t e) {
        for (int64_t sid = b; sid < e; ++sid) {
            const CSlot s = t.slot((uint32_t)sid);
            if (!enabled || s.ref == 0xffffffffu) continue;
            float c[3], rad;
            compat_extent(s, c, rad);
            if (rad <= 0.5f * R) est[sid] = compat_refine(t, c[0], c[1], c[2], R, k, iters);
        }
    });
    parallel_for_blocks(nq, 64, nthreads, [&](int64_t b, int64_t e) {
        for (int64_t q = b; q < e; ++q) {
            const float qx = q4[4 * q], qy = q4[4 * q + 1], qz = q4[4 * q + 2];
            float est_q = R;
            uint32_t sid = 0;
            for (int depth = 0; depth < 4096; ++depth) {
                const CSlot s = t.slot(sid);
                if (s.ref == 0xffffffffu) break;
                float c[3], rad;
                compat_extent(s, c, rad);
                const float len = std::sqrt(d2_f32(qx, qy, qz, c[0], c[1], c[2]));
                est_q = std::min(est_q, len + est[sid]);
                if (s.cnt > 0) break;
                const CSlot s0 = t.slot(s.ref << 1), s1 = t.slot((s.ref << 1) | 1u);
                const float b0 = s0.ref == 0xffffffffu ? INFINITY : box_lb_f32(qx, qy, qz, s0.lo, s0.hi);
                const float b1 = s1.ref == 0xffffffffu ? INFINITY : box_lb_f32(qx, qy, qz, s1.lo, s1.hi);
                sid = (s.ref << 1) | (b1 < b0 ? 1u : 0u);
            }
            const float r = compat_refine(t, qx, qy, qz, est_q, k, iters);
            out_radius[q] = r;
            if (!out_rad) continue;
            const float r2 = r * r;
            uint32_t count = 0;
            float maxd2 = 0.0f;
            compat_range(t, qx, qy, qz, r2, [&](uint32_t, float d2) { ++count; maxd2 = std::max(maxd2, d2); });
            const float r2u = count >= k ? maxd2 : r2;
            out_count[q] = count;
            out_r2[q] = r2u;
            double acc[3] = {0, 0, 0};
            if (count > 0 && count >= min_found && r2u > 0.0f) {
                const double r2d = r2u, kc = cone_k;
                compat_range(t, qx, qy, qz, r2, [&](uint32_t i, float) {
                    if (!front_f32(n4[4 * q], n4[4 * q + 1], n4[4 * q + 2], f2u(tpow4[4 * (size_t)i + 3]))) return;
                    const double dx = (double)tpos4[4 * (size_t)i] - qx, dy = (double)tpos4[4 * (size_t)i + 1] - qy,
                                 dz = (double)tpos4[4 * (size_t)i + 2] - qz;
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    double w = 1.0;
                    if (filter == 1) w = 1.0 - std::sqrt(d2) / (kc * std::sqrt(r2d));
                    else if (filter == 2) w = 1.0 - d2 / r2d;
                    for (int c = 0; c < 3; ++c) acc[c] += w * (double)tpow4[4 * (size_t)i + c];
                });
                double norm = 1.0 / (kPi * r2d);
                if (filter == 1) norm = 1.0 / ((1.0 - 2.0 / (3.0 * kc)) * kPi * r2d);
                else if (filter == 2) norm = 2.0 / (kPi * r2d);
                for (int c = 0; c < 3; ++c) acc[c] *= norm;
            }
            for (int c = 0; c < 3; ++c) out_rad[3 * q + c] = acc[c];
        }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Illumination cuts restated on the engine's exported tree (slot 0 = root,
// slots 2j and 2j + 1 = children of internal node j), following
// PhotonMap::OnFinalNodeList / GenerateFinalIllumCut (PhotonMap.cpp:287-452),
// the kernels of GPU/illumcut.cu and dev_InterpolateNodeIrradiance
// (GPU/photon_knn.cu:338-433), with the engine's stated choices: slots are the
// tree nodes; a slot's photon sums run lane-strided over 32 partial sums
// combined by the butterfly 16, 8, 4, 2, 1; the level mean is an exact 64-bit
// fixed-point sum (scale 2^40 / largest |E~|); the refinement's race between
// "finished" and "re-added by the parent" resolves to re-added; interpolation
// visits the slots whose box lies within R.  The cover pass below is the
// reference's literal top-down level loop (illumcut.cu:384-440).
namespace {

constexpr uint32_t kIcutLimit = 5000;   // ICUT_PHOTONLIMIT, illumcut.cu:74
constexpr uint32_t kInv = 0xffffffffu;

float butterfly32(float p[32]) {
    for (int o = 16; o; o >>= 1) {
        float q[32];
        for (int l = 0; l < 32; ++l) q[l] = p[l] + p[l ^ o];
        std::memcpy(p, q, sizeof(q));
    }
    return p[0];
}

inline float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    float a = ax * bx, b = ay * by, c = az * bz;
    float s = a + b;
    return s + c;
}

void icut_range(const CompatTree& t, uint32_t sid, uint32_t* first, uint32_t* end) {
    const CSlot s = t.slot(sid);
    if (s.cnt > 0) { first[sid] = s.ref; end[sid] = s.ref + s.cnt; return; }
    const uint32_t a = s.ref << 1, b = a | 1u;
    icut_range(t, a, first, end);
    icut_range(t, b, first, end);
    first[sid] = std::min(first[a], first[b]);
    end[sid] = std::max(end[a], end[b]);
}

}  // namespace

extern "C" {

// Slot records: level (kInv for empty slots), photon range [first, end),
// centre xyz + largest side (center4).
void orc_icut_slots(const uint32_t* nodes, uint32_t m, uint32_t* level, uint32_t* first, uint32_t* end,
                    float* center4) {
    CompatTree t{nodes, m, nullptr, nullptr};
    const uint32_t ns = 2 * (m + 1);
    for (uint32_t s = 0; s < ns; ++s) {
        level[s] = kInv; first[s] = end[s] = 0;
        for (int a = 0; a < 4; ++a) center4[4 * s + a] = 0.0f;
    }
    if (t.slot(0).ref == kInv) return;
    icut_range(t, 0, first, end);
    std::vector<std::pair<uint32_t, uint32_t>> stack{{0u, 0u}};
    while (!stack.empty()) {
        const auto [sid, lvl] = stack.back();
        stack.pop_back();
        const CSlot s = t.slot(sid);
        level[sid] = lvl;
        float e[3];
        for (int a = 0; a < 3; ++a) {
            e[a] = s.hi[a] - s.lo[a];
            center4[4 * sid + a] = s.lo[a] + 0.5f * e[a];
        }
        center4[4 * sid + 3] = std::max(e[0], std::max(e[1], e[2]));
        if (s.cnt == 0) {
            stack.push_back({s.ref << 1, lvl + 1});
            stack.push_back({(s.ref << 1) | 1u, lvl + 1});
        }
    }
}

// Normal per slot from its photons (normalised sum of -d/|d|), slots of
// fewer than 5,000 photons; zero otherwise.
void orc_icut_normals(const float* tpow4, uint32_t ns, const uint32_t* first, const uint32_t* end, float* normal4) {
    for (uint32_t s = 0; s < ns; ++s) {
        float p[3][32] = {{0}};
        const uint32_t cnt = end[s] - first[s];
        if (cnt > 0 && cnt < kIcutLimit) {
            for (uint32_t i = first[s]; i < end[s]; ++i) {
                const int l = (int)((i - first[s]) & 31u);
                float d[3];
                oct_decode(f2u(tpow4[4 * (size_t)i + 3]), d);
                const float len = std::sqrt(dot3(d[0], d[1], d[2], d[0], d[1], d[2]));
                if (len > 0.0f)
                    for (int a = 0; a < 3; ++a) p[a][l] = p[a][l] - d[a] / len;
            }
        }
        float v[3];
        for (int a = 0; a < 3; ++a) v[a] = butterfly32(p[a]);
        const float l = std::sqrt(dot3(v[0], v[1], v[2], v[0], v[1], v[2]));
        for (int a = 0; a < 3; ++a) normal4[4 * s + a] = l > 0.0f ? v[a] / l : 0.0f;
        normal4[4 * s + 3] = 0.0f;
    }
}

// Photon-sum estimate E~ = sum(front * flux) / side^2 (illumcut.cu:151-209).
void orc_icut_estimate(const float* tpow4, uint32_t ns, const uint32_t* first, const uint32_t* end,
                       const float* center4, const float* normal4, float* est4) {
    for (uint32_t s = 0; s < ns; ++s) {
        const float* n = normal4 + 4 * s;
        const uint32_t cnt = end[s] - first[s];
        const bool eval = cnt > 0 && cnt < kIcutLimit && dot3(n[0], n[1], n[2], n[0], n[1], n[2]) > 0.0f;
        float p[3][32] = {{0}};
        if (eval) {
            for (uint32_t i = first[s]; i < end[s]; ++i) {
                const int l = (int)((i - first[s]) & 31u);
                const float* w = tpow4 + 4 * (size_t)i;
                if (front_f32(n[0], n[1], n[2], f2u(w[3])))
                    for (int a = 0; a < 3; ++a) p[a][l] = p[a][l] + w[a];
            }
        }
        float v[3];
        for (int a = 0; a < 3; ++a) v[a] = butterfly32(p[a]);
        const float side = center4[4 * s + 3];
        const bool ok = eval && side > 0.0f;
        const float a2 = side * side;
        for (int a = 0; a < 3; ++a) est4[4 * s + a] = ok ? v[a] / a2 : 0.0f;
        est4[4 * s + 3] = 0.0f;
    }
}

// Coarse cut: every leaf, or E_min marks -> remove parents -> cover pass.
// emin_out (3 floats, may be NULL) receives E_min.
void orc_icut_coarse(const uint32_t* nodes, uint32_t m, const uint32_t* level, const float* est4, int use_leafs,
                     uint32_t level_emin, uint32_t* coarse, float* emin_out) {
    CompatTree t{nodes, m, nullptr, nullptr};
    const uint32_t ns = 2 * (m + 1);
    if (use_leafs) {
        for (uint32_t s = 0; s < ns; ++s) {
            const CSlot c = t.slot(s);
            coarse[s] = (c.ref != kInv && c.cnt > 0) ? 1u : 0u;
        }
        return;
    }
    // E_min: mean of the nonzero estimates on level_emin (illumcut.cu:587-625)
    float mx[3] = {0, 0, 0};
    uint64_t count = 0;
    auto on_level = [&](uint32_t s) {
        const float* e = est4 + 4 * s;
        return level[s] == level_emin && !(e[0] == 0.0f && e[1] == 0.0f && e[2] == 0.0f);
    };
    for (uint32_t s = 0; s < ns; ++s) {
        if (!on_level(s)) continue;
        ++count;
        for (int a = 0; a < 3; ++a) mx[a] = std::max(mx[a], std::fabs(est4[4 * s + a]));
    }
    double scale[3];
    int64_t sum[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a) scale[a] = mx[a] > 0.0f ? 1099511627776.0 / (double)mx[a] : 0.0;
    for (uint32_t s = 0; s < ns; ++s) {
        if (!on_level(s)) continue;
        for (int a = 0; a < 3; ++a) sum[a] += (int64_t)std::llrint((double)est4[4 * s + a] * scale[a]);
    }
    float emin[3];
    for (int a = 0; a < 3; ++a) {
        if (count == 0) emin[a] = INFINITY;
        else if (scale[a] == 0.0) emin[a] = 0.0f;
        else emin[a] = (float)(((double)sum[a] / scale[a]) / (double)count);
        if (emin_out) emin_out[a] = emin[a];
    }
    std::vector<uint32_t> mark0(ns), mark(ns), covered(ns, 0u);
    uint32_t max_level = 0;
    for (uint32_t s = 0; s < ns; ++s) {
        const float* e = est4 + 4 * s;
        mark0[s] = (level[s] != kInv && e[0] >= emin[0] && e[1] >= emin[1] && e[2] >= emin[2]) ? 1u : 0u;
        if (level[s] != kInv) max_level = std::max(max_level, level[s]);
    }
    // kernel_RemoveParents (illumcut.cu:352-370)
    for (uint32_t s = 0; s < ns; ++s) {
        mark[s] = mark0[s];
        const CSlot c = t.slot(s);
        if (c.ref != kInv && c.cnt == 0) {
            const uint32_t l = mark0[2 * c.ref], r = mark0[2 * c.ref + 1];
            if ((l == 1 && r == 1) || (l == 0 && r == 0)) mark[s] = 0;
        }
    }
    // kernel_UpdateCoveredState, level by level from the root (illumcut.cu:384-440)
    for (uint32_t lvl = 0; lvl <= max_level; ++lvl) {
        for (uint32_t s = 0; s < ns; ++s) {
            if (level[s] != lvl) continue;
            const CSlot c = t.slot(s);
            uint32_t my_mark = mark[s];
            if (c.cnt > 0) {
                if (covered[s] == 0) my_mark = 1;
            } else {
                const uint32_t l = 2 * c.ref, r = l + 1;
                uint32_t ml = mark[l], mr = mark[r], cl, cr;
                if (covered[s] == 1) { ml = 0; mr = 0; cl = 1; cr = 1; }
                else { cl = ml; cr = mr; }
                mark[l] = ml; mark[r] = mr; covered[l] = cl; covered[r] = cr;
            }
            mark[s] = my_mark;
        }
    }
    for (uint32_t s = 0; s < ns; ++s) coarse[s] = level[s] != kInv ? mark[s] : 0u;
}

// Final cut from the coarse cut (illumcut.cu:488-519, PhotonMap.cpp:387-452).
void orc_icut_final(const uint32_t* nodes, uint32_t m, const uint32_t* coarse, const float* est4, const float* exact4,
                    uint32_t iters, float accuracy, uint32_t* fin) {
    CompatTree t{nodes, m, nullptr, nullptr};
    const uint32_t ns = 2 * (m + 1);
    std::vector<uint32_t> work(coarse, coarse + ns), next(ns);
    for (uint32_t s = 0; s < ns; ++s) fin[s] = 0;
    for (uint32_t it = 0; it < iters; ++it) {
        if (std::none_of(work.begin(), work.end(), [](uint32_t w) { return w != 0; })) break;
        std::fill(next.begin(), next.end(), 0u);
        for (uint32_t s = 0; s < ns; ++s) {
            if (!work[s]) continue;
            const CSlot c = t.slot(s);
            if (c.ref == kInv) continue;
            const float* a = est4 + 4 * s;
            const float* b = exact4 + 4 * s;
            bool ok = true;
            for (int k = 0; k < 3; ++k) ok = ok && std::fabs(a[k] - b[k]) < accuracy * b[k];
            ok = ok || c.cnt > 0;
            if (ok) fin[s] = 1;
            else { next[2 * c.ref] = 1; next[2 * c.ref + 1] = 1; }
        }
        work.swap(next);
    }
    for (uint32_t s = 0; s < ns; ++s)
        if (work[s]) fin[s] = 1;
}

// Interpolation at queries (dev_InterpolateNodeIrradiance, photon_knn.cu:
// 338-433): out (3 nq doubles), reached (nq, cut slots of nonzero weight).
void orc_icut_interp(const uint32_t* nodes, uint32_t m, const uint32_t* fin, const float* center4,
                     const float* normal4, const float* exact4, const float* q4, const float* n4, uint32_t nq,
                     float R, double* out, uint32_t* reached, int nthreads) {
    CompatTree t{nodes, m, nullptr, nullptr};
    const float r2 = R * R;
    parallel_for_blocks(nq, 64, nthreads, [&](int64_t b, int64_t e) {
        for (int64_t q = b; q < e; ++q) {
            const float qx = q4[4 * q], qy = q4[4 * q + 1], qz = q4[4 * q + 2];
            const float* qn = n4 + 4 * q;
            double acc[3] = {0, 0, 0}, ws = 0.0;
            uint32_t nr = 0;
            std::vector<uint32_t> stack{0u};
            while (!stack.empty()) {
                const uint32_t sid = stack.back();
                stack.pop_back();
                const CSlot s = t.slot(sid);
                if (s.ref == kInv || !(box_lb_f32(qx, qy, qz, s.lo, s.hi) < r2)) continue;
                if (s.cnt == 0 && !fin[sid]) {
                    stack.push_back(s.ref << 1);
                    stack.push_back((s.ref << 1) | 1u);
                    continue;
                }
                const float* nn = normal4 + 4 * sid;
                if (dot3(nn[0], nn[1], nn[2], nn[0], nn[1], nn[2]) == 0.0f) continue;
                const float* c = center4 + 4 * sid;
                const float dist = std::sqrt(d2_f32(qx, qy, qz, c[0], c[1], c[2]));
                if (!(c[3] > 0.0f)) continue;
                const float tt = dist / c[3];
                const float rbf = tt <= 1.0f ? 1.0f - tt * tt : 0.0f;
                const float w = rbf * std::max(0.0f, dot3(nn[0], nn[1], nn[2], qn[0], qn[1], qn[2]));
                if (w == 0.0f) continue;
                ++nr;
                for (int a = 0; a < 3; ++a) acc[a] += (double)w * (double)exact4[4 * sid + a];
                ws += (double)w;
            }
            for (int a = 0; a < 3; ++a) out[3 * q + a] = ws != 0.0 ? acc[a] / ws : 0.0;
            reached[q] = nr;
        }
    });
}

}  // extern "C"
