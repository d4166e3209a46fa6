/*
 * pmgpu.hpp -- C++ classes shaped like the reference's PhotonMap and
 * KDTreePoint (jonike/mnrt PhotonMap.h:89-257, KDTreePoint.h:83-160), over
 * the C ABI of pmgpu.h, so that callers written against the reference port
 * one to one.  Header only; link with libpmgpu.so and the CUDA runtime.
 *
 * Differences from the reference, by design:
 *   - the kNN is exact (PM_MODE_EXACT) unless SetModeCompat(true) selects the
 *     reference's histogram radius pipeline;
 *   - errors throw pmgpu::Error instead of aborting (MNFatal);
 *   - every call runs on the stream given to SetStream (default: legacy
 *     default stream, as the reference);
 *   - Merge returns the merged count like the reference and is synchronous.
 */
#ifndef PMGPU_HPP
#define PMGPU_HPP

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "pmgpu.h"

namespace pmgpu {

typedef unsigned int uint;

/* The reference's data records at the boundary (KernelDefs.h:160-291,
 * 537-629; RayPool.h:162-178): only the fields the photon map reads. */
struct PhotonData {
    float4* d_positions = nullptr;   /* xyz, w = azimuth (reference layout) */
    float4* d_powers = nullptr;      /* rgb flux, w = polar angle */
    uint numPhotons = 0;
    uint maxPhotons = 0;
};

struct ShadingPoints {
    uint numPoints = 0;
    float4* d_ptInter = nullptr;     /* hit positions */
    float4* d_normalsS = nullptr;    /* shading normals */
};

struct RayChunk {
    uint numRays = 0;
    float4* d_origins = nullptr;
    float4* d_dirs = nullptr;
    float4* d_influences = nullptr;
};

class Error : public std::runtime_error {
public:
    Error(pm_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    pm_status status;
};

inline void check(pm_status s, const pm_map* m) {
    if (s != PM_OK) throw Error(s, std::string(m ? pm_last_error(m) : pm_status_string(s)));
}

/* PhotonMap (PhotonMap.h:89-257). */
class PhotonMap {
public:
    /* PhotonMap(maxPhotons, sceneAABBMin, sceneAABBMax, globalQRadiusMax, settings) */
    PhotonMap(uint maxPhotons, float3 sceneAABBMin, float3 sceneAABBMax, float globalQRadiusMax,
              int photonFormat = PM_PHOTONS_REFERENCE)
        : m_rMax(globalQRadiusMax), m_format(photonFormat) {
        const float lo[3] = {sceneAABBMin.x, sceneAABBMin.y, sceneAABBMin.z};
        const float hi[3] = {sceneAABBMax.x, sceneAABBMax.y, sceneAABBMax.z};
        check(pm_create(&m_map, maxPhotons, lo, hi, globalQRadiusMax), nullptr);
    }
    ~PhotonMap() { if (m_map) pm_destroy(m_map); }
    PhotonMap(const PhotonMap&) = delete;
    PhotonMap& operator=(const PhotonMap&) = delete;

    /* Merge (PhotonMap.cpp:181): appends the valid photons of other. */
    uint Merge(const PhotonData& other, uint* d_isValid) {
        uint merged = 0;
        check(pm_merge(m_map, reinterpret_cast<const float*>(other.d_positions),
                       reinterpret_cast<const float*>(other.d_powers), d_isValid, other.numPhotons, &merged, m_stream),
              m_map);
        return merged;
    }
    /* ScaleFlux (PhotonMap.cpp:186): RGB flux only. */
    void ScaleFlux(float scale) {
        uint n = 0;
        pm_merged_count(m_map, &n);
        if (n == 0 && !m_built) return;   /* nothing to do, as the reference */
        check(pm_scale_flux(m_map, scale, m_stream), m_map);
    }
    /* BuildMap (PhotonMap.cpp:157-171): the point kd-tree over the merged
     * photons, then the illumination cut when cuts are enabled. */
    bool BuildMap() {
        check(pm_build_merged(m_map, m_format, m_stream), m_map);
        m_built = true;
        uint n = 0;
        pm_merged_count(m_map, &n);
        if (m_useICut && n > 0) {
            pm_query_desc d = Desc(m_k, m_rMax);
            check(pm_icut_build(m_map, &m_icut, &d, nullptr, m_stream), m_map);
        }
        return true;
    }
    /* Clears the merged photons (PhotonData::Clear). */
    void Clear() { check(pm_clear_merged(m_map), m_map); }

    /* Gather (PhotonMap.cpp:195): estimate at the shading points themselves
     * (never from the illumination cut, :206-224). */
    void Gather(const ShadingPoints& sp, const RayChunk& rayChunk, float4* d_clrDiffHit, float4* d_ioRadiance) {
        pm_query_desc d = Desc(m_k, m_rMax);
        check(pm_gather_for(m_map, &d, F(sp.d_ptInter), F(sp.d_normalsS), F(rayChunk.d_dirs), F(rayChunk.d_origins),
                            F(rayChunk.d_influences), F(d_clrDiffHit), nullptr, sp.numPoints,
                            reinterpret_cast<float*>(d_ioRadiance), nullptr, m_stream),
              m_map);
    }
    /* GatherFor (PhotonMap.cpp:234): final-gather accumulation, from the
     * illumination cut when cuts are enabled (:244-257). */
    void GatherFor(const ShadingPoints& sp, const RayChunk& rayChunk, float4* d_clrDiffHit, uint* d_idxShadingPts,
                   float4* d_ioRadiance, float* d_ioReciDistAccu) {
        pm_query_desc d = Desc(m_k, m_rMax);
        if (m_useICut) d.mode = PM_MODE_ICUT;
        check(pm_gather_for(m_map, &d, F(sp.d_ptInter), F(sp.d_normalsS), F(rayChunk.d_dirs), F(rayChunk.d_origins),
                            F(rayChunk.d_influences), F(d_clrDiffHit), d_idxShadingPts, sp.numPoints,
                            reinterpret_cast<float*>(d_ioRadiance), d_ioReciDistAccu, m_stream),
              m_map);
    }
    /* Visualize (PhotonMap.cpp:272): nearest photon within 5 % of the radius. */
    void Visualize(const ShadingPoints& sp, const RayChunk& rayChunk, float4* d_ioRadiance) {
        pm_query_desc d = Desc(1, m_rMax * 0.05f);
        d.min_found = 0;
        check(pm_gather_for(m_map, &d, F(sp.d_ptInter), F(sp.d_normalsS), F(rayChunk.d_dirs), F(rayChunk.d_origins),
                            F(rayChunk.d_influences), nullptr, nullptr, sp.numPoints,
                            reinterpret_cast<float*>(d_ioRadiance), nullptr, m_stream),
              m_map);
    }

    void SetKNNTargetCount(uint k) { m_k = k; }           /* PhotonMap.h:257 */
    uint GetKNNTargetCount() const { return m_k; }
    float GetGlobalQRadiusMax() const { return m_rMax; }
    uint GetPhotonCount() const {
        pm_map_info info;
        check(pm_get_info(m_map, &info, m_stream), m_map);
        return info.num_photons;
    }
    void SetStream(cudaStream_t s) { m_stream = s; }
    void SetModeCompat(bool on) { m_mode = on ? PM_MODE_ZHOU_COMPAT : PM_MODE_EXACT; }
    /* MNRTSettings::SetUseIllumCuts and the ICut* settings (MNRTSettings.h:491-523). */
    void SetUseIllumCuts(bool on) { m_useICut = on; }
    void SetICutParams(bool useLeafs, uint levelEmin, uint refineIters, float accuracy) {
        m_icut.use_leafs = useLeafs ? 1 : 0;
        m_icut.level_emin = levelEmin;
        m_icut.refine_iters = refineIters;
        m_icut.accuracy = accuracy;
    }
    void SetFilter(int filter, float coneK = 1.0f) { m_filter = filter; m_coneK = coneK; }
    pm_map* Handle() const { return m_map; }

private:
    pm_query_desc Desc(uint k, float r) const {
        pm_query_desc d;
        d.k = k; d.r_max = r; d.filter = m_filter; d.cone_k = m_coneK; d.mode = m_mode;
        d.min_found = 8;   /* GPU/photon_knn.cu:518-519 */
        d.order = PM_ORDER_SORTED; d.refine_iters = 2;
        return d;
    }
    static const float* F(const float4* p) { return reinterpret_cast<const float*>(p); }

    pm_map* m_map = nullptr;
    float m_rMax;
    int m_format;
    uint m_k = 100;                  /* PhotonMap.cpp:111 */
    int m_mode = PM_MODE_EXACT;
    int m_filter = PM_FILTER_BOX;    /* the reference's filter */
    float m_coneK = 1.0f;
    bool m_built = false;
    bool m_useICut = false;
    pm_icut_desc m_icut = {1, 12, 4, 0.2f};   /* MNRTSettings defaults */
    cudaStream_t m_stream = nullptr;
};

/* KDTreePoint (KDTreePoint.h:83-160): a point kd-tree over arbitrary points
 * (the reference also builds it over cluster centres, RTCore.cpp:988-1004),
 * with the reference's query radius estimate. */
class KDTreePoint {
public:
    KDTreePoint(float4* d_points, uint numPoints, float3 sceneAABBMin, float3 sceneAABBMax, float maxQueryRadius)
        : m_points(d_points), m_n(numPoints), m_rMax(maxQueryRadius) {
        const float lo[3] = {sceneAABBMin.x, sceneAABBMin.y, sceneAABBMin.z};
        const float hi[3] = {sceneAABBMax.x, sceneAABBMax.y, sceneAABBMax.z};
        check(pm_create(&m_map, numPoints, lo, hi, maxQueryRadius), nullptr);
    }
    ~KDTreePoint() {
        if (m_zero) cudaFree(m_zero);
        if (m_map) pm_destroy(m_map);
    }
    KDTreePoint(const KDTreePoint&) = delete;
    KDTreePoint& operator=(const KDTreePoint&) = delete;

    /* BuildTree (KDTreeGPU.cpp:175): points carry no flux. */
    bool BuildTree() {
        if (m_n && !m_zero) {
            if (cudaMalloc(&m_zero, (size_t)m_n * sizeof(float4)) != cudaSuccess ||
                cudaMemsetAsync(m_zero, 0, (size_t)m_n * sizeof(float4), m_stream) != cudaSuccess)
                throw Error(PM_ERR_OOM, "KDTreePoint: no memory for the point records");
        }
        check(pm_build(m_map, reinterpret_cast<const float*>(m_points), static_cast<const float*>(m_zero), m_n,
                       PM_PHOTONS_PACKED, m_stream),
              m_map);
        return true;
    }
    /* ComputeQueryRadii (KDTreePoint.cpp:229): the reference's histogram radius. */
    void ComputeQueryRadii(float4* d_queryPoints, uint numQueryPoints, float* d_outRadii) {
        pm_query_desc d;
        d.k = m_k; d.r_max = m_rMax; d.filter = PM_FILTER_BOX; d.cone_k = 1.0f; d.mode = PM_MODE_ZHOU_COMPAT;
        d.min_found = 0; d.order = PM_ORDER_AS_GIVEN; d.refine_iters = m_iters;
        check(pm_compute_query_radii(m_map, &d, reinterpret_cast<const float*>(d_queryPoints), numQueryPoints, d_outRadii,
                                     m_stream),
              m_map);
    }
    void SetKNNTargetCount(uint k) { m_k = k; }
    void SetKNNRefineIters(uint iters) { m_iters = iters; }
    float GetMaxQueryRadius() const { return m_rMax; }
    void SetStream(cudaStream_t s) { m_stream = s; }
    pm_map* Handle() const { return m_map; }

private:
    pm_map* m_map = nullptr;
    float4* m_points;
    uint m_n;
    float m_rMax;
    uint m_k = 100;
    uint m_iters = 2;   /* MNRTSettings.h:443 */
    void* m_zero = nullptr;
    cudaStream_t m_stream = nullptr;
};

}  // namespace pmgpu

#endif /* PMGPU_HPP */
