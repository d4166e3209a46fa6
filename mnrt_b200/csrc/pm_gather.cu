// pm_gather.cu -- final-gather accumulation around the exact-kNN estimate.
//
// Restates the post-processing of kernel_PhotonGather (GPU/photon_knn.cu:
// 493-551) as reached from PhotonMap::GatherFor (PhotonMap.cpp:234-270):
//   * the shading normal is flipped to face the incoming gather ray
//     (dot(-dir, n) < 0 -> n = -n, :504-505);
//   * the estimate E at the hit (the engine's exact-kNN query with the
//     flipped normal; estimates from fewer than min_found photons are zeroed
//     when a diffuse colour is given, :518-519);
//   * optionally recip[idx] += rsqrt(|hit - origin|^2)            (:529-535);
//   * radiance[idx] += clr.w * clr.rgb * (1/pi) * E * influence.rgb (:540-550),
//     idx = idx_shading[i] or i.
// Like the reference, the accumulation uses no atomics: indices must be
// distinct within one call (one gather ray per shading point).
#include "pm_internal.h"

namespace pm {

namespace {

__global__ void k_gather_normals(const float4* __restrict__ hit_nrm, const float4* __restrict__ ray_dir, uint32_t n,
                                 float4* __restrict__ out_nrm) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 nn = hit_nrm[i];
    const float4 d = ray_dir[i];
    // dot(-dir, n) with a fixed evaluation order
    const float dt = __fadd_rn(__fadd_rn(__fmul_rn(-d.x, nn.x), __fmul_rn(-d.y, nn.y)), __fmul_rn(-d.z, nn.z));
    out_nrm[i] = dt < 0.0f ? make_float4(-nn.x, -nn.y, -nn.z, 0.0f) : make_float4(nn.x, nn.y, nn.z, 0.0f);
}

__global__ void k_gather_accum(const float4* __restrict__ est, const float4* __restrict__ hit_pos,
                               const float4* __restrict__ ray_origin, const float4* __restrict__ influence,
                               const float4* __restrict__ clr_diffuse, const uint32_t* __restrict__ idx_shading,
                               uint32_t n, float4* __restrict__ io_rad, float* __restrict__ io_recip) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t idx = idx_shading ? idx_shading[i] : i;
    if (io_recip) {
        const float4 h = hit_pos[i], o = ray_origin[i];
        const float dx = __fsub_rn(h.x, o.x), dy = __fsub_rn(h.y, o.y), dz = __fsub_rn(h.z, o.z);
        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        io_recip[idx] = __fadd_rn(io_recip[idx], __frsqrt_rn(d2));
    }
    const float4 c = clr_diffuse ? clr_diffuse[i] : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    const float4 e = est[i];
    const float4 f = influence[i];
    const float inv_pi = 0.318309886183790671538f;
    const float rx = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(c.w, c.x), inv_pi), e.x), f.x);
    const float ry = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(c.w, c.y), inv_pi), e.y), f.y);
    const float rz = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(c.w, c.z), inv_pi), e.z), f.z);
    float4 r = io_rad[idx];
    r.x = __fadd_rn(r.x, rx);
    r.y = __fadd_rn(r.y, ry);
    r.z = __fadd_rn(r.z, rz);
    io_rad[idx] = r;
}

}  // namespace

int gather_normals(const float4* hit_nrm, const float4* ray_dir, uint32_t n, float4* out_nrm, cudaStream_t st) {
    if (!n) return 0;
    k_gather_normals<<<(n + 255) / 256, 256, 0, st>>>(hit_nrm, ray_dir, n, out_nrm);
    return 1;
}

int gather_accumulate(const float4* est, const float4* hit_pos, const float4* ray_origin, const float4* influence,
                      const float4* clr_diffuse, const uint32_t* idx_shading, uint32_t n, float4* io_rad,
                      float* io_recip, cudaStream_t st) {
    if (!n) return 0;
    k_gather_accum<<<(n + 255) / 256, 256, 0, st>>>(est, hit_pos, ray_origin, influence, clr_diffuse, idx_shading, n,
                                                    io_rad, io_recip);
    return 1;
}

}  // namespace pm

// ---- photon ingest: PhotonData::Merge (KernelDefs.cpp:363-384) ----------
namespace pm {

namespace {

__global__ void k_valid_flags(const uint32_t* __restrict__ is_valid, uint32_t n, uint32_t* __restrict__ flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = (is_valid == nullptr || is_valid[i] != 0u) ? 1u : 0u;
}

__global__ void k_merge_scatter(const float4* __restrict__ pos, const float4* __restrict__ pw,
                                const uint32_t* __restrict__ flags, const uint32_t* __restrict__ rank, uint32_t n,
                                float4* __restrict__ dst_pos, float4* __restrict__ dst_pow) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flags[i]) return;
    const uint32_t d = rank[i];
    dst_pos[d] = pos[i];
    dst_pow[d] = pw[i];
}

__global__ void k_scale_rgb(float4* __restrict__ pw, uint32_t n, float scale) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 w = pw[i];
    w.x = __fmul_rn(w.x, scale);
    w.y = __fmul_rn(w.y, scale);
    w.z = __fmul_rn(w.z, scale);
    pw[i] = w;
}

}  // namespace

// Flags -> exclusive ranks (rank[n] is not written; *total gets the count).
int merge_ranks(const uint32_t* is_valid, uint32_t n, uint32_t* flags, uint32_t* rank, uint32_t* scan_scratch,
                uint32_t* total, cudaStream_t st) {
    k_valid_flags<<<(n + 255) / 256, 256, 0, st>>>(is_valid, n, flags);
    return 1 + exclusive_scan(flags, rank, n, scan_scratch, total, st);
}

int merge_scatter(const float4* pos, const float4* pw, const uint32_t* flags, const uint32_t* rank, uint32_t n,
                  float4* dst_pos, float4* dst_pow, cudaStream_t st) {
    k_merge_scatter<<<(n + 255) / 256, 256, 0, st>>>(pos, pw, flags, rank, n, dst_pos, dst_pow);
    return 1;
}

int scale_rgb(float4* pw, uint32_t n, float scale, cudaStream_t st) {
    if (!n) return 0;
    k_scale_rgb<<<(n + 255) / 256, 256, 0, st>>>(pw, n, scale);
    return 1;
}

}  // namespace pm
