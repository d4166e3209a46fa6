// pm_common.cuh -- device-side numeric contract shared by every kernel.
//
// Every expression here is written with explicit round-to-nearest intrinsics
// so that nvcc cannot contract or reorder it; the CPU oracle evaluates the
// same expressions with -ffp-contract=off and gets the same bits.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pm {

constexpr uint32_t kMaxK = 128;        // largest k a query supports
constexpr uint32_t kLeafMax = 64;      // photons per leaf (upper bound; two per lane where a warp scans a leaf)
constexpr int kStackDepth = 128;       // traversal stack entries per warp
constexpr uint32_t kInvalid = 0xffffffffu;

// Device error bits (mirror PM_DEVERR_* in include/pmgpu.h).
constexpr uint32_t kErrStack = 0x1u;
constexpr uint32_t kErrNonFinite = 0x2u;
constexpr uint32_t kErrQueryNonFinite = 0x4u;
constexpr uint32_t kErrWait = 0x8u;        // a bounded wait gave up (the launch's results are invalid)

// Child slot of a tree node: refitted AABB of the child's photons plus a
// reference.  cnt > 0: leaf holding photons [ref, ref + cnt) in tree order;
// cnt == 0: internal node index ref; ref == kInvalid: empty slot.
struct __align__(16) ChildSlot {
    float lo[3];
    float hi[3];
    uint32_t ref;
    uint32_t cnt;
};
struct __align__(16) Node {
    ChildSlot c[2];
};
static_assert(sizeof(ChildSlot) == 32, "slot is two 16-byte words");
static_assert(sizeof(Node) == 64, "node is four 16-byte words");

// 32-wide tree over the binary one: every binary node whose depth below its
// root is a multiple of kWideLevels is a wide node; its children are the slots
// reached by expanding kWideLevels binary levels (at most 32), stored
// contiguously.  A child slot with cnt & kWideFlag references a wide node:
// ref = index of its first child slot, cnt & kWideCount = its child count.
constexpr int kWideLevels = 5;
constexpr uint32_t kWideFlag = 0x80000000u;
constexpr uint32_t kWideCount = 0x3fu;

// Per-map header kept in device memory (written by the build).
struct MapHeader {
    float lo[3];
    float hi[3];
    float max_power;
    float fix_scale;    // fix_scale_of(max_power): fixed-point scale of the kNN flux sums
    uint32_t n;
    uint32_t num_nodes; // internal nodes (excluding the super-root at index 0)
    uint32_t errors;
    uint32_t pad;
};

// ------------------------------------------------------------ arithmetic --

// Fixed-point scale of the kNN flux sums: 2^53 / max |flux| (0 without flux,
// clamped to 2^127 for tiny flux), so a term is at most 2^53 and the up to
// 128 terms of one query sum below 2^60.  The resolution, 2^-53 of the
// largest photon flux, keeps channels of very small flux exact to FP64-like
// relative precision.
constexpr float kFixOne = 9007199254740992.0f;   // 2^53
__device__ __forceinline__ float fix_scale_of(float max_power) {
    return max_power > 0.0f ? fminf(__fdiv_rn(kFixOne, max_power), 1.7014118346046923e38f) : 0.0f;
}

__device__ __forceinline__ float d2_rn(float qx, float qy, float qz, float px, float py, float pz) {
    const float dx = __fsub_rn(px, qx), dy = __fsub_rn(py, qy), dz = __fsub_rn(pz, qz);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Lower bound of d2_rn(q, p) over every p inside [lo, hi]: per-axis gap,
// squared and summed in the same order, so rounding monotonicity keeps it
// <= the FP32 distance of any point in the box.
__device__ __forceinline__ float box_lb(float qx, float qy, float qz, const float* lo, const float* hi) {
    const float gx = fmaxf(fmaxf(__fsub_rn(lo[0], qx), __fsub_rn(qx, hi[0])), 0.0f);
    const float gy = fmaxf(fmaxf(__fsub_rn(lo[1], qy), __fsub_rn(qy, hi[1])), 0.0f);
    const float gz = fmaxf(fmaxf(__fsub_rn(lo[2], qz), __fsub_rn(qz, hi[2])), 0.0f);
    return __fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz));
}

// Octahedral direction code, 16-bit snorm halves.  Decodes to an
// unnormalised vector; only its sign against a normal is used.
__device__ __forceinline__ void oct_decode(uint32_t bits, float& x, float& y, float& z) {
    const int16_t iu = (int16_t)(bits & 0xffffu), iv = (int16_t)(bits >> 16);
    const float s = 1.0f / 32767.0f;
    const float fu = __fmul_rn((float)iu, s), fv = __fmul_rn((float)iv, s);
    const float au = fabsf(fu), av = fabsf(fv);
    z = __fsub_rn(__fsub_rn(1.0f, au), av);
    x = fu;
    y = fv;
    if (z < 0.0f) {
        x = __fmul_rn(__fsub_rn(1.0f, av), fu >= 0.0f ? 1.0f : -1.0f);
        y = __fmul_rn(__fsub_rn(1.0f, au), fv >= 0.0f ? 1.0f : -1.0f);
    }
}

__device__ __forceinline__ int32_t snorm16(float f) {
    float r = rintf(__fmul_rn(f, 32767.0f));
    r = fminf(fmaxf(r, -32767.0f), 32767.0f);
    return (int32_t)r;
}

__device__ __forceinline__ uint32_t oct_encode(float dx, float dy, float dz) {
    const float s = __fadd_rn(__fadd_rn(fabsf(dx), fabsf(dy)), fabsf(dz));
    if (!(s > 0.0f)) return 0u;
    float px = __fdiv_rn(dx, s), py = __fdiv_rn(dy, s);
    if (dz < 0.0f) {
        const float ax = fabsf(px), ay = fabsf(py);
        const float nx = __fmul_rn(__fsub_rn(1.0f, ay), px >= 0.0f ? 1.0f : -1.0f);
        const float ny = __fmul_rn(__fsub_rn(1.0f, ax), py >= 0.0f ? 1.0f : -1.0f);
        px = nx;
        py = ny;
    }
    return (uint32_t)(snorm16(px) & 0xffff) | ((uint32_t)(snorm16(py) & 0xffff) << 16);
}

// Front-face test dot(n, -dir) > 0 (reference GPU/photon_knn.cu:196-208).
__device__ __forceinline__ bool front_rn(float nx, float ny, float nz, uint32_t dirbits) {
    float x, y, z;
    oct_decode(dirbits, x, y, z);
    const float a = __fmul_rn(nx, -x), b = __fmul_rn(ny, -y), c = __fmul_rn(nz, -z);
    return __fadd_rn(__fadd_rn(a, b), c) > 0.0f;
}

// Deterministic FP64 sin/cos for the spherical photon ingest: Cody-Waite
// reduction by pi/2 with a 33-bit head, then Taylor series of degree 21 (sin)
// and 22 (cos) on [-pi/4, pi/4], each step one IEEE double rounding.
__device__ __forceinline__ void sincos_det(double x, double& s_out, double& c_out) {
    const double kPio2Hi = 0x1.921fb544p+0;
    const double kPio2Lo = 0x1.0b4611a626331p-34;
    const double kTwoOverPi = 0x1.45f306dc9c883p-1;
    const double kq = rint(__dmul_rn(x, kTwoOverPi));
    const double r0 = __dsub_rn(x, __dmul_rn(kq, kPio2Hi));
    const double r = __dsub_rn(r0, __dmul_rn(kq, kPio2Lo));
    const double r2 = __dmul_rn(r, r);
    const double sc[10] = {-1.0 / 121645100408832000.0, 1.0 / 355687428096000.0, -1.0 / 1307674368000.0,
                           1.0 / 6227020800.0,          -1.0 / 39916800.0,      1.0 / 362880.0,
                           -1.0 / 5040.0,               1.0 / 120.0,            -1.0 / 6.0,
                           1.0};
    double ps = 1.0 / 51090942171709440000.0;
#pragma unroll
    for (int i = 0; i < 10; ++i) ps = __dadd_rn(__dmul_rn(ps, r2), sc[i]);
    const double sv = __dmul_rn(ps, r);
    const double cc[11] = {1.0 / 2432902008176640000.0, -1.0 / 6402373705728000.0, 1.0 / 20922789888000.0,
                           -1.0 / 87178291200.0,        1.0 / 479001600.0,         -1.0 / 3628800.0,
                           1.0 / 40320.0,               -1.0 / 720.0,              1.0 / 24.0,
                           -1.0 / 2.0,                  1.0};
    double pc = -1.0 / 1124000727777607680000.0;
#pragma unroll
    for (int i = 0; i < 11; ++i) pc = __dadd_rn(__dmul_rn(pc, r2), cc[i]);
    const double cv = pc;
    const int q = ((int)(long long)kq) & 3;
    double s, c;
    if (q == 0) { s = sv; c = cv; }
    else if (q == 1) { s = cv; c = -sv; }
    else if (q == 2) { s = -sv; c = -cv; }
    else { s = -cv; c = sv; }
    s_out = s;
    c_out = c;
}

__device__ __forceinline__ uint32_t spherical_to_oct(float phi, float theta) {
    double sp, cp, st, ct;
    sincos_det((double)phi, sp, cp);
    sincos_det((double)theta, st, ct);
    const double x = __dmul_rn(st, cp), y = __dmul_rn(st, sp);
    return oct_encode(__double2float_rn(x), __double2float_rn(y), __double2float_rn(ct));
}

// Up to 16 bits -> every third bit of 48.
__device__ __forceinline__ uint64_t spread3_16(uint32_t v) {
    uint64_t x = v & 0xffffull;
    x = (x | (x << 16)) & 0x0000ff0000ffull;
    x = (x | (x << 8)) & 0x00f00f00f00full;
    x = (x | (x << 4)) & 0x0c30c30c30c3ull;
    x = (x | (x << 2)) & 0x249249249249ull;
    return x;
}

__device__ __forceinline__ uint32_t quantize16(float v, float lo, float scale) {
    float t = __fmul_rn(__fsub_rn(v, lo), scale);
    t = fminf(fmaxf(t, 0.0f), 65535.0f);   // NaN -> 0 via fmaxf
    return (uint32_t)t;
}

// 10 bits -> every third bit of 30.
__device__ __forceinline__ uint32_t spread3_10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 30-bit Hilbert index of the top 10 bits of each axis' 16-bit quantisation:
// the order queries are processed in (coherence only; results do not depend
// on it).  Consecutive indices are face-adjacent cells, so consecutive
// queries stay close where a Morton order jumps between quadrants, and the
// radius bound each query takes from its predecessor stays tight (measured
// 7.80 -> 7.63 ms query kernel on the plain workload).  The axes-to-transpose
// step of J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707
// (2004): undo the excess work level by level, Gray-encode, then interleave
// the transposed bits (axis 0 most significant in each triple).
__device__ __forceinline__ uint32_t hilbert30(float x, float y, float z, const float* lo, float scale) {
    uint32_t X[3] = {quantize16(x, lo[0], scale) >> 6, quantize16(y, lo[1], scale) >> 6,
                     quantize16(z, lo[2], scale) >> 6};
#pragma unroll
    for (uint32_t Q = 1u << 9; Q > 1u; Q >>= 1) {
        const uint32_t P = Q - 1u;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (X[i] & Q) {
                X[0] ^= P;                              // invert the low bits of axis 0
            } else {
                const uint32_t t = (X[0] ^ X[i]) & P;   // exchange the low bits of axes 0 and i
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    uint32_t t = 0;
#pragma unroll
    for (uint32_t Q = 1u << 9; Q > 1u; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1u;
    X[0] ^= t;
    X[1] ^= t;
    X[2] ^= t;
    return (spread3_10(X[0]) << 2) | (spread3_10(X[1]) << 1) | spread3_10(X[2]);
}

// 30-bit Morton code of the same 10-bit cells (the cut interpolation's query order).
__device__ __forceinline__ uint32_t morton30(float x, float y, float z, const float* lo, float scale) {
    return (spread3_10(quantize16(x, lo[0], scale) >> 6) << 2) | (spread3_10(quantize16(y, lo[1], scale) >> 6) << 1) |
           spread3_10(quantize16(z, lo[2], scale) >> 6);
}

// Morton code of a photon in the map's cubic cell: the top 13 bits of each
// axis' 16-bit quantisation, interleaved (x most significant), 39 bits in
// all.  The tree's leaves hold up to 64 photons, far coarser than 13-bit
// cells (at the densest caustic of the benchmark workloads a cell holds about
// 5 photons), so finer codes only lengthen the sort: 5 radix passes instead of
// the 6 of 16 bits per axis.  Equal codes are ordered by caller index.
constexpr int kMortonBits = 39;
__device__ __forceinline__ uint64_t morton39(float x, float y, float z, const float* lo, float scale) {
    return (spread3_16(quantize16(x, lo[0], scale) >> 3) << 2) | (spread3_16(quantize16(y, lo[1], scale) >> 3) << 1) |
           spread3_16(quantize16(z, lo[2], scale) >> 3);
}


__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

}  // namespace pm
