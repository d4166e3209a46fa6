// Drives the C++ shim (include/pmgpu.hpp) the way reference code drives
// PhotonMap / KDTreePoint, and checks every result bit for bit against the
// same work done through the C ABI directly.  Exit code 0 = pass.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pmgpu.hpp"

namespace {

uint32_t g_state = 12345u;
float rnd() {   // xorshift32 in [0, 1)
    g_state ^= g_state << 13;
    g_state ^= g_state >> 17;
    g_state ^= g_state << 5;
    return (float)(g_state >> 8) * (1.0f / 16777216.0f);
}

template <class T>
T* to_device(const std::vector<T>& h) {
    T* d = nullptr;
    if (cudaMalloc(&d, h.size() * sizeof(T) + 16) != cudaSuccess) return nullptr;
    cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

template <class T>
std::vector<T> to_host(const T* d, size_t n) {
    std::vector<T> h(n);
    cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

int fail(const char* what) {
    std::printf("shim test FAILED: %s\n", what);
    return 1;
}

}  // namespace

int main() {
    using pmgpu::uint;
    const uint n = 40000, nq = 5000;
    // photons on the floor and the x = 0 wall, reference layout (azimuth, polar angle)
    std::vector<float4> pos(n), pw(n);
    std::vector<uint> valid(n);
    for (uint i = 0; i < n; ++i) {
        const bool floor = (i & 1u) == 0;
        const float u = rnd(), v = rnd();
        pos[i] = floor ? make_float4(u, 0.0f, v, 6.2831853f * rnd()) : make_float4(0.0f, u, v, 6.2831853f * rnd());
        pw[i] = make_float4(rnd() / n, rnd() / n, rnd() / n, 3.1415926f * rnd());
        valid[i] = (i % 3 != 0) ? 7u : 0u;   // any non-zero flag is valid
    }
    std::vector<float4> qpos(nq), qnrm(nq), ori(nq), dir(nq), infl(nq), clr(nq);
    std::vector<uint> idx(nq);
    for (uint i = 0; i < nq; ++i) {
        const bool floor = (i & 1u) == 0;
        const float u = rnd(), v = rnd();
        qpos[i] = floor ? make_float4(u, 0.0f, v, 0.0f) : make_float4(0.0f, u, v, 0.0f);
        qnrm[i] = floor ? make_float4(0.0f, 1.0f, 0.0f, 0.0f) : make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        dir[i] = floor ? make_float4(0.1f, -1.0f, 0.2f, 0.0f) : make_float4(-1.0f, 0.3f, 0.1f, 0.0f);
        ori[i] = make_float4(qpos[i].x - dir[i].x, qpos[i].y - dir[i].y, qpos[i].z - dir[i].z, 0.0f);
        infl[i] = make_float4(rnd(), rnd(), rnd(), 0.0f);
        clr[i] = make_float4(rnd(), rnd(), rnd(), 1.0f);
        idx[i] = nq - 1 - i;
    }
    float4 *d_pos = to_device(pos), *d_pw = to_device(pw);
    uint* d_valid = to_device(valid);
    float4 *d_qpos = to_device(qpos), *d_qnrm = to_device(qnrm), *d_ori = to_device(ori), *d_dir = to_device(dir);
    float4 *d_infl = to_device(infl), *d_clr = to_device(clr);
    uint* d_idx = to_device(idx);
    std::vector<float4> zero4(nq, make_float4(0, 0, 0, 0));
    std::vector<float> zero1(nq, 0.0f);
    float4 *d_rad_a = to_device(zero4), *d_rad_b = to_device(zero4);
    float *d_rec_a = to_device(zero1), *d_rec_b = to_device(zero1);
    if (!d_pos || !d_rad_b || !d_rec_b) return fail("cudaMalloc");

    // ---- the reference-shaped path
    pmgpu::PhotonData traced;
    traced.d_positions = d_pos; traced.d_powers = d_pw; traced.numPhotons = n; traced.maxPhotons = n;
    pmgpu::PhotonMap pm(n, make_float3(0, 0, 0), make_float3(1, 1, 1), 0.1f);
    const uint merged = pm.Merge(traced, d_valid);
    uint expect = 0;
    for (uint i = 0; i < n; ++i) expect += valid[i] ? 1u : 0u;
    if (merged != expect) return fail("Merge count");
    pm.ScaleFlux(0.5f);
    pm.BuildMap();
    pm.SetKNNTargetCount(50);
    if (pm.GetPhotonCount() != expect) return fail("GetPhotonCount");
    pmgpu::ShadingPoints sp;
    sp.numPoints = nq; sp.d_ptInter = d_qpos; sp.d_normalsS = d_qnrm;
    pmgpu::RayChunk rc;
    rc.numRays = nq; rc.d_origins = d_ori; rc.d_dirs = d_dir; rc.d_influences = d_infl;
    pm.GatherFor(sp, rc, d_clr, d_idx, d_rad_a, d_rec_a);

    // ---- the same through the C ABI directly (compaction and scaling on the host)
    std::vector<float4> cpos, cpw;
    for (uint i = 0; i < n; ++i)
        if (valid[i]) {
            cpos.push_back(pos[i]);
            float4 w = pw[i];
            w.x *= 0.5f; w.y *= 0.5f; w.z *= 0.5f;
            cpw.push_back(w);
        }
    float4 *d_cpos = to_device(cpos), *d_cpw = to_device(cpw);
    pm_map* raw = nullptr;
    const float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    if (pm_create(&raw, n, lo, hi, 0.1f) != PM_OK) return fail("pm_create");
    if (pm_build(raw, (const float*)d_cpos, (const float*)d_cpw, (uint32_t)cpos.size(), PM_PHOTONS_REFERENCE, nullptr) != PM_OK)
        return fail("pm_build");
    pm_query_desc d;
    d.k = 50; d.r_max = 0.1f; d.filter = PM_FILTER_BOX; d.cone_k = 1.0f; d.mode = PM_MODE_EXACT;
    d.min_found = 8; d.order = PM_ORDER_SORTED; d.refine_iters = 2;
    if (pm_gather_for(raw, &d, (const float*)d_qpos, (const float*)d_qnrm, (const float*)d_dir, (const float*)d_ori,
                      (const float*)d_infl, (const float*)d_clr, d_idx, nq, (float*)d_rad_b, d_rec_b, nullptr) != PM_OK)
        return fail("pm_gather_for");
    cudaDeviceSynchronize();
    const std::vector<float4> ra = to_host(d_rad_a, nq), rb = to_host(d_rad_b, nq);
    const std::vector<float> ca = to_host(d_rec_a, nq), cb = to_host(d_rec_b, nq);
    if (std::memcmp(ra.data(), rb.data(), nq * sizeof(float4)) != 0) return fail("GatherFor radiance");
    if (std::memcmp(ca.data(), cb.data(), nq * sizeof(float)) != 0) return fail("GatherFor reciprocal distances");
    bool any = false;
    for (const float4& r : ra) any = any || r.x > 0.0f;
    if (!any) return fail("GatherFor produced no radiance");

    // ---- GatherFor from the illumination cut (MNRTSettings' default: cuts on,
    // the leaves as the coarse cut), against the same calls on the C ABI
    pmgpu::PhotonMap pmc(n, make_float3(0, 0, 0), make_float3(1, 1, 1), 0.1f);
    pmc.SetUseIllumCuts(true);
    pmc.SetKNNTargetCount(50);
    pmc.Merge(traced, d_valid);
    pmc.ScaleFlux(0.5f);
    pmc.BuildMap();
    float4 *d_rad_c = to_device(zero4), *d_rad_d = to_device(zero4);
    float *d_rec_c = to_device(zero1), *d_rec_d = to_device(zero1);
    pmc.GatherFor(sp, rc, d_clr, d_idx, d_rad_c, d_rec_c);
    pm_icut_desc cd;
    cd.use_leafs = 1; cd.level_emin = 12; cd.refine_iters = 4; cd.accuracy = 0.2f;
    if (pm_icut_build(raw, &cd, &d, nullptr, nullptr) != PM_OK) return fail("pm_icut_build");
    pm_query_desc di = d;
    di.mode = PM_MODE_ICUT;
    if (pm_gather_for(raw, &di, (const float*)d_qpos, (const float*)d_qnrm, (const float*)d_dir, (const float*)d_ori,
                      (const float*)d_infl, (const float*)d_clr, d_idx, nq, (float*)d_rad_d, d_rec_d, nullptr) != PM_OK)
        return fail("pm_gather_for (PM_MODE_ICUT)");
    cudaDeviceSynchronize();
    const std::vector<float4> rc_ = to_host(d_rad_c, nq), rd_ = to_host(d_rad_d, nq);
    if (std::memcmp(rc_.data(), rd_.data(), nq * sizeof(float4)) != 0) return fail("GatherFor (cut) radiance");
    bool any_cut = false;
    for (const float4& r : rc_) any_cut = any_cut || r.x > 0.0f;
    if (!any_cut) return fail("GatherFor (cut) produced no radiance");

    // ---- KDTreePoint over the photon positions: the reference's radius estimate
    float* d_radii_a = to_device(zero1);
    float* d_radii_b = to_device(zero1);
    pmgpu::KDTreePoint kd(d_pos, n, make_float3(0, 0, 0), make_float3(1, 1, 1), 0.1f);
    kd.SetKNNTargetCount(20);
    kd.BuildTree();
    kd.ComputeQueryRadii(d_qpos, nq, d_radii_a);
    pm_map* raw2 = nullptr;
    std::vector<float4> zpw(n, make_float4(0, 0, 0, 0));
    float4* d_zpw = to_device(zpw);
    pm_create(&raw2, n, lo, hi, 0.1f);
    pm_build(raw2, (const float*)d_pos, (const float*)d_zpw, n, PM_PHOTONS_PACKED, nullptr);
    pm_query_desc dz = d;
    dz.k = 20; dz.mode = PM_MODE_ZHOU_COMPAT; dz.min_found = 0; dz.order = PM_ORDER_AS_GIVEN;
    if (pm_compute_query_radii(raw2, &dz, (const float*)d_qpos, nq, d_radii_b, nullptr) != PM_OK)
        return fail("pm_compute_query_radii");
    cudaDeviceSynchronize();
    const std::vector<float> xa = to_host(d_radii_a, nq), xb = to_host(d_radii_b, nq);
    if (std::memcmp(xa.data(), xb.data(), nq * sizeof(float)) != 0) return fail("ComputeQueryRadii");
    for (float r : xa)
        if (!(r > 0.0f && r <= 0.1f)) return fail("ComputeQueryRadii range");

    // errors surface as exceptions, not aborts
    try {
        pmgpu::PhotonMap bad(10, make_float3(0, 0, 0), make_float3(1, 1, 1), -1.0f);
        return fail("invalid radius accepted");
    } catch (const pmgpu::Error&) {
    }
    pm_destroy(raw);
    pm_destroy(raw2);
    std::printf("shim test ok: %u photons merged, %u gathers\n", merged, nq);
    return 0;
}
