// pm_backward.cu -- reverse-mode adjoint of the exact-kNN radiance estimate.
//
// The reference has no adjoint; the forward it differentiates is the
// estimate of GPU/photon_knn.cu:113-235 (E = norm(r^2) * sum front * w * flux,
// r^2 = d^2 of the k-th neighbour when k were found, else R^2) with the
// engine's filters.  For query q, channel c and neighbour p:
//
//   E_qc   = norm(r2_q) * S_qc,   S_qc = sum_p f_qp * w(d2_qp, r2_q) * Phi_pc
//   dL/dPhi_pc  = sum_q g_qc * norm_q * f_qp * w_qp                  (exact, linear)
//   dL/dx_p     = sum_q 2 (x_p - q) * [ f_qp * (sum_c g_qc norm_q Phi_pc) * dw/dd2
//                                      + [p is the k-th of q] * G_q ]
//   G_q         = sum_c g_qc * (dnorm/dr2 * S_qc + norm_q * sum_p f_qp Phi_pc dw/dr2)
//
// The k-th neighbour moves r^2 = d2(q, x_k), which feeds every weight and the
// normalisation of q; that is the G_q path.  Set changes (a photon entering or
// leaving N(q)) are measure-zero kinks and contribute nothing.
//
// Scatter without float atomics, deterministic by construction:
//   1. k_bwd_count  warp per query: counts every photon's pairs (the
//                   listed neighbours of queries with cnt >= max(1,
//                   min_found); the per-photon pass skips the pairs of
//                   queries that carry no gradient)
//   2. exclusive scan of the counts: every photon's segment [start, end)
//   3. k_bwd_prep   warp per query: FP64 S, T sums over the neighbour list
//                   -> per-query record (g * norm, G, the filter's
//                   reciprocal, position, normal), and every pair's value
//                   (query << 1 | the photon is the query's k-th) put into
//                   its photon's segment at an atomic cursor
//   4. k_bwd_segsort warp per photon: sorts its segment's values (bitonic
//                   network in registers up to 256 values; longer segments
//                   by a block each, k_bwd_segsort_long), which restores
//                   the query order the cursor lost: the segment then holds
//                   exactly what a stable sort of the pairs by photon gives
//   5. k_bwd_reduce thread per photon: walks its segment in order and sums
//                   the FP64 contributions; the running sum carries across
//                   query chunks, so chunked and single-pass runs give the
//                   same bits
// A chunk with more than kBwdPlaceMaxFanIn pairs per photon on average
// replaces steps 1-4 by the sort path: k_bwd_prep<false> writes one (photon,
// value) pair per neighbour slot, a stable LSD radix sort orders them by
// photon and k_bwd_bounds finds the segments.  There the cursors of the
// photons that neighbouring warps share contend and the segments grow long,
// while the sort's cost does not depend on how the pairs spread; both paths
// give the same segments, so the same bits.
// Contributions are evaluated in FP64 from the FP32 inputs (the neighbour set
// and the front test follow the FP32 forward contract).
#include "pm_internal.h"

namespace pm {

namespace {

constexpr double kPiD = 3.14159265358979323846;

__device__ __forceinline__ double norm_of(int filter, double r2, double cone_k) {
    if (filter == 1) return 1.0 / ((1.0 - 2.0 / (3.0 * cone_k)) * kPiD * r2);
    if (filter == 2) return 2.0 / (kPiD * r2);
    return 1.0 / (kPiD * r2);
}

// The filter's reciprocal of one query (one FP64 division per query, none
// per neighbour pair): 1 / (k_c r) for the cone, 1 / r^2 for Epanechnikov,
// 1 for the box (a positive marker of a query that carries gradient).
__device__ __forceinline__ double filter_rinv(int filter, double r2, double cone_k) {
    if (filter == 1) return 1.0 / (cone_k * sqrt(r2));
    if (filter == 2) return 1.0 / r2;
    return 1.0;
}

// w and dw/dd2 of the filters (FP64) from the query's reciprocal rinv:
//   cone:         w = 1 - d rinv,     dw/dd2 = -rinv / (2 d)  (d = d^2 / sqrt(d^2) by one rsqrt)
//   Epanechnikov: w = 1 - d^2 rinv,   dw/dd2 = -rinv
// and dw/dr2 (the per-query pass only; inv_r2 = 1 / r^2):
//   cone: d rinv inv_r2 / 2,   Epanechnikov: d^2 rinv^2.
__device__ __forceinline__ void weight_terms(int filter, double d2, double rinv, double inv_r2, double& w,
                                             double& dw_dd2, double& dw_dr2) {
    if (filter == 1) {   // cone: w = 1 - d / (k_c r)
        const double rs = d2 > 0.0 ? rsqrt(d2) : 0.0, d = d2 * rs;
        w = 1.0 - d * rinv;
        dw_dd2 = -0.5 * rinv * rs;
        dw_dr2 = 0.5 * d * rinv * inv_r2;
    } else if (filter == 2) {   // Epanechnikov: w = 1 - d^2 / r^2
        w = 1.0 - d2 * rinv;
        dw_dd2 = -rinv;
        dw_dr2 = d2 * rinv * rinv;
    } else {   // box
        w = 1.0;
        dw_dd2 = 0.0;
        dw_dr2 = 0.0;
    }
}

__device__ __forceinline__ double dist2_d(const float4& a, const float4& b) {
    const double dx = (double)a.x - (double)b.x, dy = (double)a.y - (double)b.y, dz = (double)a.z - (double)b.z;
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The head of one query, shared by the counting pass and the per-query pass
// so that both take the same pairs: the neighbours found (the count output,
// else the valid prefix of the row), r^2 (d^2 of the k-th when k were found,
// else R^2) and whether the query carries gradient.
struct BwdHead {
    float4 qp;
    double r2;
    uint32_t cnt;
    bool active;
};

// Neighbours found by query ql: the count output, else the valid prefix of
// its row (warp-wide).
__device__ __forceinline__ uint32_t bwd_found(const BwdArgs& a, uint32_t ql, uint32_t lane) {
    const uint32_t k = a.k;
    uint32_t c = 0;
    if (a.count_in) {
        c = a.count_in[ql];
    } else {
        const uint32_t* row = a.nbr + (size_t)ql * k;
        for (uint32_t j = lane; j < k; j += 32) c += row[j] != kInvalid ? 1u : 0u;
#pragma unroll
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    return c < k ? c : k;
}

// The pairs that go into the photons' segments: every listed neighbour of a
// query with cnt >= max(1, min_found).  A superset of the pairs that carry
// gradient (the per-photon pass skips those of queries whose record has no
// filter reciprocal), decided without the query's position or r^2.
__device__ __forceinline__ bool bwd_placed(const BwdArgs& a, uint32_t cnt) { return cnt > 0 && cnt >= a.min_found; }

__device__ __forceinline__ BwdHead bwd_head(const BwdArgs& a, uint32_t ql, uint32_t q, uint32_t lane) {
    const uint32_t k = a.k;
    const uint32_t* row = a.nbr + (size_t)ql * k;
    BwdHead h;
    h.cnt = bwd_found(a, ql, lane);
    h.qp = a.qpos[q];
    h.r2 = (double)a.r_max * (double)a.r_max;
    if (h.cnt == k) h.r2 = dist2_d(a.pos[a.inv[row[k - 1]]], h.qp);
    h.active = h.cnt > 0 && h.cnt >= a.min_found && h.r2 > 0.0 && isfinite(h.qp.x) && isfinite(h.qp.y) &&
               isfinite(h.qp.z);
    return h;
}

// Warp per query, in caller order: one count per placed pair on its
// photon's cursor (the cursors are cleared before; the scan then turns the
// counts into segment starts).  Two dependent loads per pair (row, inverse
// permutation) and no per-query gathers: the pass is latency-bound.
__global__ void __launch_bounds__(256) k_bwd_count(BwdArgs a, uint32_t q0, uint32_t nq_chunk) {
    (void)q0;
    const uint32_t ql = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (ql >= nq_chunk) return;
    const uint32_t cnt = bwd_found(a, ql, lane);
    if (!bwd_placed(a, cnt)) return;
    const uint32_t* row = a.nbr + (size_t)ql * a.k;
    for (uint32_t j = lane; j < cnt; j += 32) atomicAdd(&a.cursor[a.inv[row[j]]], 1u);
}

// One warp per query of the chunk, taken in Hilbert order when a.order is
// set: neighbouring warps then gather neighbouring photons, which L1 and L2
// serve (1M queries, k = 64: 1.48 -> 1.26 ms).  Records stay at the caller's
// index and every pair's value names the caller's index, so the results do
// not depend on the order.  The warp puts each pair's value into its
// photon's segment at the photon's cursor (the segment start after the scan);
// the cursor ends at the segment's end.  The slot is taken before the FP64
// math, so the atomic's latency overlaps it.
// kPlace false (the sort path, for chunks of high fan-in): every neighbour
// slot writes its photon key (the sentinel n for a slot without a pair, which
// sorts after every photon) and value at the caller's pair index instead.
// Five blocks per SM (48 registers, a few spilled): 40 warps hide the
// dependent gathers better than 32 at 64 registers (1M x 1M, k = 64: adjoint
// 2.98 -> 2.88 ms).
template <bool kPlace>
__global__ void __launch_bounds__(256, 5) k_bwd_prep(BwdArgs a, uint32_t q0, uint32_t nq_chunk) {
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp_global >= nq_chunk) return;
    const uint32_t ql = a.order ? a.order[warp_global] : warp_global, q = q0 + ql;
    const uint32_t k = a.k;
    const uint32_t* row = a.nbr + (size_t)ql * k;
    const BwdHead h = bwd_head(a, ql, q, lane);
    const float4 qp = h.qp;
    const float4 qn = a.qnrm[q];
    const double r2 = h.r2;
    const bool active = h.active;
    const uint32_t cnt = h.cnt;
    double S0 = 0, S1 = 0, S2 = 0, T0 = 0, T1 = 0, T2 = 0;
    const double rinv = filter_rinv(a.filter, r2, (double)a.cone_k), inv_r2 = 1.0 / r2;
    const uint32_t jend = bwd_placed(a, cnt) ? cnt : 0u;
    const uint64_t pair0 = (uint64_t)ql * k;
    for (uint32_t j = lane; j < (kPlace ? jend : k); j += 32) {
        const uint32_t val = (ql << 1) | (j == k - 1 ? 1u : 0u);   // the query, and whether p is its k-th
        if (!kPlace && j >= jend) {
            a.keys[pair0 + j] = a.n;
            a.vals[pair0 + j] = val;
            continue;
        }
        const uint32_t p = a.inv[row[j]];
        const uint32_t slot = kPlace ? atomicAdd(&a.cursor[p], 1u) : 0u;
        const float4 pp = a.pos[p], pw = a.pow[p];
        if (active && front_rn(qn.x, qn.y, qn.z, __float_as_uint(pw.w))) {
            double w, dwd, dwr;
            weight_terms(a.filter, dist2_d(pp, qp), rinv, inv_r2, w, dwd, dwr);
            S0 += w * pw.x; S1 += w * pw.y; S2 += w * pw.z;
            T0 += dwr * pw.x; T1 += dwr * pw.y; T2 += dwr * pw.z;
        }
        if (kPlace) {
            if (slot < a.pair_cap) a.vals[slot] = val;
        } else {
            a.keys[pair0 + j] = p;
            a.vals[pair0 + j] = val;
        }
    }
    S0 = warp_sum_d(S0); S1 = warp_sum_d(S1); S2 = warp_sum_d(S2);
    T0 = warp_sum_d(T0); T1 = warp_sum_d(T1); T2 = warp_sum_d(T2);
    if (lane != 0) return;
    BwdQuery rec;
    rec.gx = rec.gy = rec.gz = rec.G = 0.0;
    rec.rinv = active ? rinv : 0.0;
    rec.qx = qp.x; rec.qy = qp.y; rec.qz = qp.z;
    rec.nx = qn.x; rec.ny = qn.y; rec.nz = qn.z;
    if (active) {
        const float4 g = a.grad[q];
        const double nrm = norm_of(a.filter, r2, (double)a.cone_k);
        rec.gx = (double)g.x * nrm;
        rec.gy = (double)g.y * nrm;
        rec.gz = (double)g.z * nrm;
        if (cnt == k) {
            const double dn = -nrm / r2;
            rec.G = (double)g.x * (dn * S0 + nrm * T0) + (double)g.y * (dn * S1 + nrm * T1) +
                    (double)g.z * (dn * S2 + nrm * T2);
        }
    }
    a.qrec[ql] = rec;
}

// Ascending bitonic network over the 32 R slots of a warp, slot lane R + r in
// v[r] (the all-ascending form: the first step of every merge compares a slot
// with its mirror in the block, i ^ (kk - 1), the others i with i ^ j).
template <int R>
__device__ __forceinline__ void warp_bitonic(uint32_t (&v)[R], uint32_t lane) {
#pragma unroll
    for (int kk = 2; kk <= 32 * R; kk <<= 1) {
#pragma unroll
        for (int j = kk / 2; j > 0; j >>= 1) {
            const bool flip = j == kk / 2;
            if ((flip ? kk - 1 : j) < R) {   // partner in the same lane
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int o = flip ? (r ^ (kk - 1)) : (r ^ j);
                    if (o > r) {
                        const uint32_t lo = min(v[r], v[o]), hi = max(v[r], v[o]);
                        v[r] = lo;
                        v[o] = hi;
                    }
                }
            } else {   // partner in lane ^ lm; the lower slot keeps the minimum
                const int lm = flip ? kk / R - 1 : j / R;
                const bool lower = (lane & (uint32_t)(flip ? kk / (2 * R) : j / R)) == 0;
                uint32_t w[R];
#pragma unroll
                for (int r = 0; r < R; ++r) w[r] = __shfl_xor_sync(0xffffffffu, v[flip ? R - 1 - r : r], lm);
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = lower ? min(v[r], w[r]) : max(v[r], w[r]);
            }
        }
    }
}

template <int R>
__device__ __forceinline__ void sort_segment_regs(uint32_t* seg, uint32_t m, uint32_t lane) {
    uint32_t v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t i = lane * R + r;
        v[r] = i < m ? seg[i] : 0xffffffffu;   // padding sorts last
    }
    warp_bitonic<R>(v, lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t i = lane * R + r;
        if (i < m) seg[i] = v[r];
    }
}

constexpr uint32_t kSegRegMax = 256;       // values a warp sorts in registers
constexpr uint32_t kSegSmemMax = 8192;     // values a block sorts in shared memory
constexpr int kSegLongThreads = 512;

// The all-ascending network over P (a power of two >= m) slots by a block:
// pairs (i, partner) with bit j of i clear, the slots at and above m read as
// +infinity (a pair whose upper slot is past m is already in order).  kShared:
// s is the block's shared copy; else s is the segment, sorted in place
// through L2.
template <bool kShared>
__device__ __forceinline__ void block_bitonic(uint32_t* s, uint32_t m, uint32_t P) {
    for (uint32_t lk = 1; (1u << lk) <= P; ++lk) {
        const uint32_t kk = 1u << lk;
        for (int lj = (int)lk - 1; lj >= 0; --lj) {
            const uint32_t j = 1u << lj;
            for (uint32_t t = threadIdx.x; t < (P >> 1); t += blockDim.x) {
                const uint32_t i = ((t >> lj) << (lj + 1)) | (t & (j - 1));   // bit j of i clear
                const uint32_t o = j == (kk >> 1) ? (i ^ (kk - 1)) : (i + j);
                if (o < m) {
                    const uint32_t x = kShared ? s[i] : __ldcg(s + i), y = kShared ? s[o] : __ldcg(s + o);
                    if (x > y) {
                        if (kShared) {
                            s[i] = y;
                            s[o] = x;
                        } else {
                            __stcg(s + i, y);
                            __stcg(s + o, x);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Warp per photon: sorts the values of its segment (distinct: a photon is
// in a query's list at most once), so the segment lists its queries in
// caller order.  Segments above kSegRegMax values are listed for
// k_bwd_segsort_long.
__global__ void __launch_bounds__(256, 8) k_bwd_segsort(const uint32_t* __restrict__ start,
                                                        const uint32_t* __restrict__ end, uint32_t n,
                                                        uint64_t cap, uint32_t* __restrict__ vals,
                                                        uint32_t* __restrict__ long_list,
                                                        uint32_t* __restrict__ long_count) {
    const uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (p >= n) return;
    const uint32_t e = (uint32_t)min((uint64_t)end[p], cap), b = min(start[p], e), m = e - b;
    if (m < 2) return;
    uint32_t* seg = vals + b;
    if (m <= 32) sort_segment_regs<1>(seg, m, lane);
    else if (m <= 64) sort_segment_regs<2>(seg, m, lane);
    else if (m <= 128) sort_segment_regs<4>(seg, m, lane);
    else if (m <= kSegRegMax) sort_segment_regs<8>(seg, m, lane);
    else if (lane == 0) long_list[atomicAdd(long_count, 1u)] = p;   // at most n photons: the list holds n
}

// Block per listed segment (above kSegRegMax values): in shared memory up to
// kSegSmemMax values, in place through L2 beyond.  The grid loops over the
// list, whose length only the device knows.
__global__ void __launch_bounds__(kSegLongThreads) k_bwd_segsort_long(const uint32_t* __restrict__ long_list,
                                                                      const uint32_t* __restrict__ long_count,
                                                                      const uint32_t* __restrict__ start,
                                                                      const uint32_t* __restrict__ end, uint64_t cap,
                                                                      uint32_t* __restrict__ vals) {
    __shared__ uint32_t s[kSegSmemMax];
    const uint32_t count = *long_count;
    for (uint32_t li = blockIdx.x; li < count; li += gridDim.x) {
        const uint32_t p = long_list[li];
        const uint32_t e = (uint32_t)min((uint64_t)end[p], cap), b = min(start[p], e), m = e - b;
        uint32_t* seg = vals + b;
        uint32_t P = 1;
        while (P < m) P <<= 1;
        if (m <= kSegSmemMax) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s[i] = seg[i];
            __syncthreads();
            block_bitonic<true>(s, m, P);
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) seg[i] = s[i];
        } else {
            block_bitonic<false>(seg, m, P);
        }
        __syncthreads();   // s is reused by the block's next segment
    }
}

// Sort path: segment bounds of every photon in the sorted keys (start = end
// = 0 when the photon has no pair; both arrays are cleared before).
__global__ void k_bwd_bounds(const uint32_t* __restrict__ keys, uint64_t m, uint32_t n, uint32_t* __restrict__ start,
                             uint32_t* __restrict__ end) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t key = keys[i];
    if (key >= n) return;
    if (i == 0 || keys[i - 1] != key) start[key] = (uint32_t)i;
    if (i + 1 == m || keys[i + 1] != key) end[key] = (uint32_t)(i + 1);
}

int key_bits_for(uint32_t n) {
    int b = 1;
    while (b < 32 && (1ull << b) <= (uint64_t)n) ++b;   // sentinel n must fit
    return b;
}

// One thread per photon (tree position).  acc holds 6 doubles per photon
// between chunks.
__global__ void k_bwd_reduce(BwdArgs a, uint32_t q0, const uint32_t* __restrict__ sorted_vals,
                             const uint32_t* __restrict__ start, const uint32_t* __restrict__ end, int first, int last,
                             double* __restrict__ acc, float4* __restrict__ grad_pow, float4* __restrict__ grad_pos) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    double g0 = 0, g1 = 0, g2 = 0, x0 = 0, x1 = 0, x2 = 0;
    if (!first) {
        const double* s = acc + (size_t)p * 6;
        g0 = s[0]; g1 = s[1]; g2 = s[2]; x0 = s[3]; x1 = s[4]; x2 = s[5];
    }
    const uint32_t e = (uint32_t)min((uint64_t)end[p], a.pair_cap), b = start[p];   // the cap: pair slots held
    if (b < e) {
        const float4 pp = a.pos[p], pw = a.pow[p];
        const uint32_t dir = __float_as_uint(pw.w);
        // software pipeline: the next entry's record and the value after it
        // load while this entry's math runs (the sums keep their order)
        uint32_t vnext = sorted_vals[b];   // query << 1 | (the photon is the query's k-th)
        BwdQuery rnext = a.qrec[vnext >> 1];
        uint32_t vafter = b + 1 < e ? sorted_vals[b + 1] : 0u;
        for (uint32_t i = b; i < e; ++i) {
            const uint32_t v = vnext;
            const BwdQuery rec = rnext;
            if (i + 1 < e) {
                vnext = vafter;
                rnext = a.qrec[vafter >> 1];
                vafter = i + 2 < e ? sorted_vals[i + 2] : 0u;
            }
            const double rinv = rec.rinv;
            if (!(rinv > 0.0)) continue;
            const double dx = (double)pp.x - (double)rec.qx, dy = (double)pp.y - (double)rec.qy,
                         dz = (double)pp.z - (double)rec.qz;
            const double d2 = dx * dx + dy * dy + dz * dz;
            double coef = 0.0;
            if (front_rn(rec.nx, rec.ny, rec.nz, dir)) {
                double w, dwd, dwr;
                weight_terms(a.filter, d2, rinv, 0.0, w, dwd, dwr);   // dw/dr2 is the per-query pass's
                g0 += w * rec.gx;
                g1 += w * rec.gy;
                g2 += w * rec.gz;
                coef = (rec.gx * pw.x + rec.gy * pw.y + rec.gz * pw.z) * dwd;
            }
            if (v & 1u) coef += rec.G;   // the k-th neighbour sets r^2 of q
            x0 += 2.0 * coef * dx;
            x1 += 2.0 * coef * dy;
            x2 += 2.0 * coef * dz;
        }
    }
    if (last) {
        const uint32_t caller = __float_as_uint(a.pos[p].w);
        if (grad_pow) grad_pow[caller] = make_float4((float)g0, (float)g1, (float)g2, 0.0f);
        if (grad_pos) grad_pos[caller] = make_float4((float)x0, (float)x1, (float)x2, 0.0f);
    } else {
        double* s = acc + (size_t)p * 6;
        s[0] = g0; s[1] = g1; s[2] = g2; s[3] = x0; s[4] = x1; s[5] = x2;
    }
}

}  // namespace

size_t bwd_scratch_words(uint32_t n, uint64_t pairs, bool sort_path) {
    const size_t scan = scan_scratch_words(n) + 1;
    const size_t sort = sort_path ? sort_scratch_words((uint32_t)pairs) + 64 : 0;
    return scan > sort ? scan : sort;
}

int backward_chunk(const BwdArgs& a, uint32_t q0, uint32_t nq_chunk, bool first, bool last, const BwdBuffers& b,
                   float4* grad_pow, float4* grad_pos, cudaStream_t st) {
    int nl = 0;
    BwdArgs x = a;
    const uint64_t pairs = (uint64_t)nq_chunk * a.k;
    x.pair_cap = pairs;
    const uint32_t warps_per_block = 8;
    const uint32_t qblocks = (nq_chunk + warps_per_block - 1) / warps_per_block;
    const uint32_t* sorted_vals = b.vals[0];
    if (nq_chunk > 0 && bwd_sort_path(pairs, a.n)) {
        // high fan-in: a stable radix sort of the (photon, value) pairs, whose
        // cost does not depend on how many pairs one photon holds
        x.keys = b.keys[0];
        x.vals = b.vals[0];
        x.cursor = nullptr;
        k_bwd_prep<false><<<qblocks, 32 * warps_per_block, 0, st>>>(x, q0, nq_chunk);
        ++nl;
        uint32_t* keys[2] = {b.keys[0], b.keys[1]};
        uint32_t* vals[2] = {b.vals[0], b.vals[1]};
        const int cur = radix_sort_pairs32(keys, vals, (uint32_t)pairs, key_bits_for(a.n), b.scratch, st, &nl);
        cudaMemsetAsync(b.seg_start, 0, (size_t)a.n * sizeof(uint32_t), st);
        cudaMemsetAsync(b.seg_end, 0, (size_t)a.n * sizeof(uint32_t), st);
        k_bwd_bounds<<<(uint32_t)((pairs + 255) / 256), 256, 0, st>>>(keys[cur], pairs, a.n, b.seg_start, b.seg_end);
        ++nl;
        sorted_vals = vals[cur];
    } else {
        x.keys = nullptr;
        x.vals = b.vals[0];
        x.cursor = b.seg_end;
        cudaMemsetAsync(b.seg_end, 0, (size_t)a.n * sizeof(uint32_t), st);
        if (nq_chunk > 0) {
            k_bwd_count<<<qblocks, 32 * warps_per_block, 0, st>>>(x, q0, nq_chunk);
            ++nl;
        }
        // counts -> segment starts; the cursors start there and end at the ends
        nl += exclusive_scan(b.seg_end, b.seg_end, a.n, b.scratch, nullptr, st);
        cudaMemcpyAsync(b.seg_start, b.seg_end, (size_t)a.n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
        if (nq_chunk > 0) {
            k_bwd_prep<true><<<qblocks, 32 * warps_per_block, 0, st>>>(x, q0, nq_chunk);
            cudaMemsetAsync(b.long_count, 0, sizeof(uint32_t), st);
            k_bwd_segsort<<<(a.n + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(
                b.seg_start, b.seg_end, a.n, x.pair_cap, b.vals[0], b.long_list, b.long_count);
            k_bwd_segsort_long<<<a.n < 1024u ? a.n : 1024u, kSegLongThreads, 0, st>>>(
                b.long_list, b.long_count, b.seg_start, b.seg_end, x.pair_cap, b.vals[0]);
            nl += 3;
        }
    }
    if (a.n > 0) {
        k_bwd_reduce<<<(a.n + 127) / 128, 128, 0, st>>>(x, q0, sorted_vals, b.seg_start, b.seg_end, first ? 1 : 0,
                                                        last ? 1 : 0, b.acc, grad_pow, grad_pos);
        ++nl;
    }
    return nl;
}

}  // namespace pm
