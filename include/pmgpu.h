/*
 * pmgpu.h -- C ABI of the B200 photon-map density-estimation engine.
 *
 * One engine object (pm_map) replaces the reference's PhotonMap + KDTreePoint
 * pair (paths inside jonike/mnrt):
 *   PhotonMap::PhotonMap(maxPhotons, aabbMin, aabbMax, rMax, settings)  PhotonMap.h:89
 *   PhotonMap::Merge / ScaleFlux / BuildMap                             PhotonMap.h:122-158
 *   KDTreePoint(d_points, n, aabbMin, aabbMax, rMax) + BuildTree()       KDTreePoint.h:83, KDTreeGPU.h:207
 *   PhotonMap::Gather / GatherFor / Visualize                           PhotonMap.h:195-232
 *   PhotonMap::SetKNNTargetCount                                         PhotonMap.h:257
 *   KDTreePoint::ComputeQueryRadii                                       KDTreePoint.h:122
 *
 * Conventions
 *   - Every entry point returns pm_status: 0 on success, a negative code on
 *     error.  Nothing aborts the process.  pm_last_error() describes the last
 *     failure of a handle.
 *   - "float4 arrays" are plain float pointers to 4*n contiguous floats,
 *     16-byte aligned, in device memory unless the name says host.
 *   - stream is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls are asynchronous on that stream unless documented otherwise.
 *   - Handles are independent; there is no global mutable state.  One handle
 *     must not be used from two host threads at once.
 *
 * Photon formats accepted by pm_build (PM_PHOTONS_*):
 *   REFERENCE: the reference's PhotonData (KernelDefs.h:537-629):
 *              pos.xyz = position, pos.w = azimuth phi in [0, 2pi),
 *              pow.xyz = RGB flux, pow.w = polar theta in [0, pi];
 *              incident direction = (sin t cos p, sin t sin p, cos t)
 *              (GPU/mncudautil_dev.h:345-352).
 *   PACKED:    pos.xyz = position, pos.w ignored,
 *              pow.xyz = RGB flux, pow.w = octahedral direction code
 *              (uint32 bits: 16-bit snorm u | 16-bit snorm v << 16).
 */
#ifndef PMGPU_H
#define PMGPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PM_API __attribute__((visibility("default")))
#else
#define PM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int pm_status;

enum {
    PM_OK = 0,
    PM_ERR_INVALID = -1,     /* bad argument (null pointer, k == 0, r_max <= 0, ...) */
    PM_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    PM_ERR_OOM = -3,         /* device allocation failed */
    PM_ERR_STATE = -4,       /* call not valid in this state (no map built, capture growth) */
    PM_ERR_DEVICE = -5,      /* a kernel reported an error (stack overflow, NaN input, ...) */
    PM_ERR_UNSUPPORTED = -6  /* parameter outside what this build supports (k > PM_MAX_K, 2^31 or more
                                photons or queries in one call) */
};

enum { PM_PHOTONS_REFERENCE = 0, PM_PHOTONS_PACKED = 1 };
enum { PM_FILTER_BOX = 0, PM_FILTER_CONE = 1, PM_FILTER_EPANECHNIKOV = 2 };
enum { PM_MODE_EXACT = 0, PM_MODE_ZHOU_COMPAT = 1,
       PM_MODE_ICUT = 2   /* pm_gather_for only: interpolate the map's illumination cut */ };
enum { PM_ORDER_SORTED = 0, PM_ORDER_AS_GIVEN = 1 };

/* Largest k the query kernels support. */
#define PM_MAX_K 128u

/* Device-side error bits, returned in pm_map_info.device_errors. */
#define PM_DEVERR_STACK 0x1u     /* traversal stack overflow (query result invalid) */
#define PM_DEVERR_NONFINITE 0x2u /* non-finite photon position at build */
#define PM_DEVERR_QNONFINITE 0x4u/* non-finite query position */
#define PM_DEVERR_WAIT 0x8u      /* a bounded inter-block wait gave up (that call's results are invalid) */

typedef struct pm_map pm_map;

typedef struct pm_query_desc {
    uint32_t k;          /* neighbours per query, 1..PM_MAX_K (reference: SetKNNTargetCount, default 100) */
    float r_max;         /* maximum query radius R (reference: globalQRadiusMax) */
    int filter;          /* PM_FILTER_* */
    float cone_k;        /* cone filter constant k_c >= 1 (Jensen 2001), used by PM_FILTER_CONE */
    int mode;            /* PM_MODE_EXACT or PM_MODE_ZHOU_COMPAT (PM_MODE_ICUT: pm_gather_for only) */
    uint32_t min_found;  /* estimates from fewer photons are zeroed (reference uses 8) */
    int order;           /* PM_ORDER_SORTED: sort the queries along a Hilbert curve first; AS_GIVEN: keep order */
    uint32_t refine_iters; /* ZHOU_COMPAT only: histogram refinement rounds (reference default 2) */
} pm_query_desc;

typedef struct pm_map_info {
    uint32_t num_photons;
    uint32_t num_nodes;       /* internal nodes of the tree (valid after a synchronising call) */
    uint32_t leaf_size;       /* maximum photons per leaf */
    uint32_t device_errors;   /* PM_DEVERR_* bits seen since the last pm_clear_errors */
    float bounds_min[3];
    float bounds_max[3];
    float max_power;
    uint64_t launches;        /* kernels launched through this handle so far */
} pm_map_info;

/* Allocation hook: lets a caller route engine allocations through its own
 * allocator (and lets tests inject failures).  alloc returns 0 on success. */
typedef int (*pm_alloc_fn)(void** ptr, size_t bytes, void* user);
typedef void (*pm_free_fn)(void* ptr, void* user);

/* PhotonMap::PhotonMap(maxPhotons, sceneAABBMin, sceneAABBMax, globalQRadiusMax)
 * (PhotonMap.h:89).  Makes no CUDA call; storage is reserved on first build.
 * aabb_min/aabb_max (host, 3 floats each, may be NULL) are the scene bounds;
 * the build uses the photons' own bounds, clipped to nothing. */
PM_API pm_status pm_create(pm_map** out, uint32_t max_photons, const float* aabb_min, const float* aabb_max,
                    float r_max);
PM_API pm_status pm_destroy(pm_map* map);

/* Routes this handle's device allocations through alloc/free (NULL, NULL
 * restores cudaMalloc/cudaFree).  Must be set before the first build.  Blocks
 * must be at least 16-byte aligned (cudaMalloc gives 256); a misaligned block
 * is freed again and the call fails with PM_ERR_INVALID. */
PM_API pm_status pm_set_allocator(pm_map* map, pm_alloc_fn alloc, pm_free_fn free_fn, void* user);

/* k-buffer layouts of the query kernel. */
enum { PM_KBUF_HEAP = 0,   /* one lane per query, max-heap in shared memory */
       PM_KBUF_GROUP = 1,  /* a group of lanes per query, candidate buffer + exact selection */
       PM_KBUF_WIDE = 2    /* one query per warp over the 32-wide tree, candidate buffer + exact selection */ };

/* Tuning knobs (chosen by the autotuner): photons per leaf (1..64), warps per
 * query block (1..8), rounds in the smallest work chunk (1..4096; warps take
 * chunks by guided self-scheduling: long chunks first, this size last), queries per warp
 * (1, 2, 4, 8; group layout) and the k-buffer layout (PM_KBUF_*). */
PM_API pm_status pm_set_tuning(pm_map* map, uint32_t leaf_size, int warps_per_block, int rounds_per_chunk,
                               int queries_per_warp, int kbuf_layout);

/* The autotuner's choice (no counterpart in the reference). */
typedef struct pm_tuning {
    uint32_t leaf_size;
    int warps_per_block;
    int rounds_per_chunk;
    int queries_per_warp;
    int kbuf_layout;
    float build_ms;          /* timed build of the chosen setting */
    float query_ms;          /* timed query of the sample, scaled to all nq queries */
} pm_tuning;

/* Times build + query over a grid of tuning candidates (leaf size, warps per
 * block, rounds per chunk, queries per warp, k-buffer layout) on a strided
 * sample of at most max_sample queries (0 = all), applies the fastest to the
 * map, writes it to *best and leaves the map built with it.  Synchronous.
 * A sample is sparser than the full set, which weakens the reuse of the
 * previous query's radius bound between Hilbert neighbours: tune on all
 * queries (or a dense spatial subset) when the setting matters. */
PM_API pm_status pm_autotune(pm_map* map, const float* d_pos4, const float* d_pow4, uint32_t n, int format,
                             const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4, uint32_t nq,
                             uint32_t max_sample, pm_tuning* best, void* stream);

/* Reserves storage for up to max_photons photons and max_queries queries so
 * that later builds and queries allocate nothing (needed for stream capture). */
PM_API pm_status pm_reserve(pm_map* map, uint32_t max_photons, uint32_t max_queries);

/* KDTreePoint(d_points, n, ...) + KDTreeGPU::BuildTree() (KDTreeGPU.cpp:175),
 * fused with PhotonMap::BuildMap (PhotonMap.cpp:157).  The engine copies and
 * reorders the photons; the caller's buffers may be reused after the call
 * completes on the stream.  n == 0 builds an empty map. */
PM_API pm_status pm_build(pm_map* map, const float* d_pos4, const float* d_pow4, uint32_t n, int format,
                   void* stream);

/* PhotonMap::Merge (PhotonMap.cpp:181-184, PhotonData::Merge
 * KernelDefs.cpp:363-384): appends the photons i with d_is_valid[i] != 0
 * (NULL = all) to the map's merged photon store, in order; *merged gets the
 * count.  Synchronous, like the reference (it returns the count).  Exceeding
 * max_photons is an error (the reference aborts). */
PM_API pm_status pm_merge(pm_map* map, const float* d_pos4, const float* d_pow4, const uint32_t* d_is_valid, uint32_t n,
                          uint32_t* merged, void* stream);
/* PhotonMap::BuildMap (PhotonMap.cpp:157) over the merged store (pm_build
 * of those photons). */
PM_API pm_status pm_build_merged(pm_map* map, int format, void* stream);
/* PhotonData::Clear (KernelDefs.cpp:333-337): empties the merged store. */
PM_API pm_status pm_clear_merged(pm_map* map);
PM_API pm_status pm_merged_count(const pm_map* map, uint32_t* count);

/* Exact-kNN radiance estimate (the kernel_PhotonGather / dev_RangeSearch path,
 * GPU/photon_knn.cu:113-235,487-552, with exact k-nearest semantics).
 *   d_qpos4, d_qnrm4: query positions and normals (float4, w ignored), nq each.
 *   d_rad4 (required): per-query irradiance estimate (rgb; w = count as float).
 *   d_nbr (optional, nq*k uint32): neighbour photon indices (caller order),
 *          sorted by (d^2, index); unused slots hold 0xFFFFFFFF.
 *   d_r2 (optional, nq floats): r^2 used by the filter.
 *   d_count (optional, nq uint32): neighbours found (<= k).
 * In PM_MODE_ZHOU_COMPAT the estimate follows the reference's own answer: a
 * histogram-refined radius, then every photon inside it (d_nbr must be NULL). */
PM_API pm_status pm_query(pm_map* map, const pm_query_desc* desc, const float* d_qpos4, const float* d_qnrm4,
                   uint32_t nq, float* d_rad4, uint32_t* d_nbr, float* d_r2, uint32_t* d_count, void* stream);

/* Build + query from host memory in one call (PhotonMap::BuildMap followed
 * by GatherFor's estimate, for a caller whose photons and shading points live
 * in host memory).  Copies the photons in and builds while the queries copy
 * in on an internal stream; with chunks > 1 (at most 16; 0 = 1) the queries
 * are copied, answered and copied back in that many pieces so that copies
 * overlap queries -- at the cost of query coherence: each piece is Hilbert
 * sorted on its own, which measured slower for 2M queries than one piece.
 * Results are identical, bit for bit, to pm_build + pm_query on the same data
 * (exact mode).  Host arrays should be pinned (cudaHostAlloc /
 * cudaHostRegister) for the copies to overlap; a pinned h_rad4 is written in
 * place by the query kernel, with no download after it.  Asynchronous on `stream`:
 * h_rad4 is complete when the stream's work up to this call is.  Not
 * allowed during stream capture. */
PM_API pm_status pm_build_query_host(pm_map* map, const float* h_pos4, const float* h_pow4, uint32_t n, int format,
                                     const pm_query_desc* desc, const float* h_qpos4, const float* h_qnrm4,
                                     uint32_t nq, float* h_rad4, uint32_t chunks, void* stream);

/* Brute-force exact kNN over every photon (test and validation path). */
PM_API pm_status pm_query_bruteforce(pm_map* map, const pm_query_desc* desc, const float* d_qpos4,
                              const float* d_qnrm4, uint32_t nq, float* d_rad4, uint32_t* d_nbr, float* d_r2,
                              uint32_t* d_count, void* stream);

/* Largest query count pm_query_noalloc accepts. */
#define PM_NOALLOC_MAX_QUERIES 262144u

/* pm_query without any device allocation.  No counterpart in the reference
 * (which allocates from its memory pool inside every gather).
 *
 * For callers that cannot allocate device memory when they query: a render
 * loop that must not stall (cudaMalloc and cudaFree synchronise the device),
 * or a host application that gives the engine a fixed memory budget and lets
 * nothing grow after start-up.  Same arguments and the same results, bit for
 * bit, as pm_query on a built map.
 *   - The map must already be built.  The caller passes every input and
 *     output buffer, as for pm_query.
 *   - The query scratch (Hilbert sort keys, the list of queries re-evaluated
 *     with FP64 distances, the work counters) lives in one fixed array of
 *     about 5.1 MiB inside this library.  Every GPU that loads
 *     the library holds it until the process exits.
 *   - nq > PM_NOALLOC_MAX_QUERIES is rejected with PM_ERR_INVALID; split
 *     larger query sets into several calls.
 *   - The first call on each device looks up the array's device address,
 *     with that device current.  Make that first call before any stream
 *     capture: a first call on a capturing stream returns PM_ERR_STATE.
 *     The address is kept for the life of the process; after
 *     cudaDeviceReset on a device, do not call this entry point there again.
 *   - pm_last_timings after this call reports its launch count but no phase
 *     times, and pm_query_stats does not count it.
 *   - Every call, on every handle and stream, shares the one array.  Calls
 *     that overlap on the GPU (two streams, two threads) race and give wrong
 *     results.  Serialise them, e.g. on one stream.
 *   - PM_MODE_ZHOU_COMPAT is not supported here (PM_ERR_UNSUPPORTED). */
PM_API pm_status pm_query_noalloc(pm_map* map, const pm_query_desc* desc, const float* d_qpos4,
                                  const float* d_qnrm4, uint32_t nq, float* d_rad4, uint32_t* d_nbr, float* d_r2,
                                  uint32_t* d_count, void* stream);

/* Reverse-mode adjoint of pm_query (exact mode; no counterpart in the
 * reference).  Given dL/dE per query (d_grad_rad4, rgb), writes dL/dpower
 * (d_grad_pow4, rgb, w = 0) and dL/dposition (d_grad_pos4, xyz, w = 0) for
 * every photon in caller order; either output may be NULL.
 *   d_nbr, d_count: the forward's neighbour lists and counts (pm_query with
 *          the same desc); d_nbr == NULL recomputes the kNN in chunks.
 *   d_r2:  not read (r^2 is re-derived in FP64 from the k-th neighbour).
 * Position gradients flow through the filter weights and through r^2, which
 * the k-th neighbour sets.  Contributions are evaluated in FP64 and summed
 * per photon in query order (pairs grouped by photon, each photon's segment
 * sorted; no float atomics): the result is bitwise reproducible, and
 * identical with or without reuse and for any chunking. */
PM_API pm_status pm_query_backward(pm_map* map, const pm_query_desc* desc, const float* d_qpos4,
                            const float* d_qnrm4, uint32_t nq, const float* d_grad_rad4, const uint32_t* d_nbr,
                            const float* d_r2, const uint32_t* d_count, float* d_grad_pow4, float* d_grad_pos4,
                            void* stream);

/* Largest number of queries one backward pass handles at once (0 =
 * automatic: up to 2^27 neighbour pairs per pass).  Smaller chunks need less
 * scratch; results do not change. */
PM_API pm_status pm_set_backward_chunk(pm_map* map, uint32_t max_queries);

/* PhotonMap::GatherFor (PhotonMap.cpp:234-270, kernel_PhotonGather
 * GPU/photon_knn.cu:493-551): estimate at gather-ray hits and accumulate
 *   d_io_radiance4[idx] += clr.w * clr.rgb / pi * E * influence.rgb
 *   d_io_recip_dist[idx] += rsqrt(|hit - origin|^2)   (if non-NULL)
 * with idx = d_idx_shading[i] (NULL = i), the normal flipped to face the
 * incoming ray, and estimates from fewer than desc->min_found photons zeroed
 * when d_clr_diffuse4 is non-NULL.  NULL d_clr_diffuse4 means white and no
 * min_found rule (the reference's photon visualisation).  Indices must be
 * distinct within one call (the reference accumulates without atomics).
 * desc->mode == PM_MODE_ICUT takes E from the map's illumination cut
 * (pm_icut_interpolate with R = desc->r_max and the normal as given;
 * kernel_InterpolateIrradiance, GPU/photon_knn.cu:598-660) instead of a
 * photon search, as the reference's GatherFor does with cuts enabled. */
PM_API pm_status pm_gather_for(pm_map* map, const pm_query_desc* desc, const float* d_hit_pos4,
                        const float* d_hit_nrm4, const float* d_ray_dir4, const float* d_ray_origin4,
                        const float* d_ray_influence4, const float* d_clr_diffuse4, const uint32_t* d_idx_shading,
                        uint32_t n, float* d_io_radiance4, float* d_io_recip_dist, void* stream);

/* ---- Illumination cuts (Wang et al. 2009 as the reference builds them:
 * PhotonMap::OnFinalNodeList / GenerateFinalIllumCut PhotonMap.cpp:287-452,
 * GPU/illumcut.cu, and the interpolation of GPU/photon_knn.cu:338-433,
 * 598-660).  A cut is a set of tree nodes with one on every root-to-leaf
 * path; irradiance is estimated once per cut node and final-gather queries
 * interpolate it (pm_gather_for with desc->mode == PM_MODE_ICUT, the
 * reference's GatherFor when MNRTSettings::GetUseIllumCuts() is set).
 *
 * The cut's nodes are the engine tree's slots: slot 0 is the root, slots
 * 2j and 2j + 1 are the two children of internal node j; slot 1 is unused.
 * A built map has 2 (num_nodes + 1) slots (pm_map_info.num_nodes). */
typedef struct pm_icut_desc {
    int use_leafs;           /* 1: the coarse cut is every leaf (MNRTSettings ICutUseLeafs, default 1) */
    uint32_t level_emin;     /* tree level whose mean estimate is E_min (ICutLevelEmin, default 12) */
    uint32_t refine_iters;   /* refinement rounds of the final cut (ICutRefineIters, default 4), <= 64 */
    float accuracy;          /* required relative accuracy of a cut node (ICutAccuracy, default 0.2) */
} pm_icut_desc;

/* Builds the cut of the current tree (PhotonMap::BuildMap with illumination
 * cuts on, PhotonMap.cpp:166-168).  node_query says how the irradiance at a
 * node centre is estimated (k, r_max, filter, min_found; PM_MODE_EXACT or
 * PM_MODE_ZHOU_COMPAT -- the reference uses the latter with the box filter
 * and min_found 8, PhotonMap.cpp:371-384).  d_node_normals4 (optional, one
 * float4 per slot, w ignored) gives the surface normal at each slot's centre;
 * the reference derives it from the scene geometry (PhotonMap.cpp:339-364).
 * Without it the engine uses the normalised sum of the reversed incident
 * directions of the slot's photons (slots of fewer than 5,000 photons; larger
 * slots get no normal and no estimate).  Synchronises the stream once (node
 * count); the rest is asynchronous.  A rebuild of the map drops the cut. */
PM_API pm_status pm_icut_build(pm_map* map, const pm_icut_desc* cut, const pm_query_desc* node_query,
                               const float* d_node_normals4, void* stream);
/* Number of slots of the built tree (synchronous). */
PM_API pm_status pm_icut_slot_count(pm_map* map, uint32_t* count);
/* Per slot: box centre (xyz) and largest box side (w), for a caller that
 * computes normals from its geometry before pm_icut_build.  Empty slots get
 * zeros. */
PM_API pm_status pm_icut_node_centers(pm_map* map, float* d_centers4, void* stream);
/* Irradiance interpolated from the cut at each query (xyz; w = cut nodes of
 * nonzero weight): every cut node reached through nodes whose box lies within r_max
 * of q contributes w = (1 - t^2) max(0, n_node . n_q), t = |centre - q| /
 * side <= 1; E = sum(w E_node) / sum(w), 0 when the weights sum to 0.  The
 * normal is used as given (the reference does not flip it here). */
PM_API pm_status pm_icut_interpolate(pm_map* map, float r_max, const float* d_qpos4, const float* d_qnrm4,
                                     uint32_t nq, float* d_irr4, void* stream);
/* Copies the cut for validation (host arrays of max_slots entries; any may be
 * NULL): coarse and final marks (0/1), levels (0xFFFFFFFF for empty slots),
 * centres (xyz, side), normals, photon-sum estimates and node-centre
 * irradiance (float4 each).  Synchronous. */
PM_API pm_status pm_icut_export(pm_map* map, uint32_t max_slots, uint32_t* h_coarse, uint32_t* h_final,
                                uint32_t* h_level, float* h_center4, float* h_normal4, float* h_est4,
                                float* h_exact4);

/* PhotonMap::ScaleFlux (PhotonMap.cpp:186-193): scales the RGB flux of the
 * photons the map holds -- the built tree and the merged store -- in place
 * (direction bits untouched). */
PM_API pm_status pm_scale_flux(pm_map* map, float scale, void* stream);

/* KDTreePoint::ComputeQueryRadii (KDTreePoint.cpp:229-248) in ZHOU_COMPAT
 * semantics: the reference's histogram-refined query radius per point. */
PM_API pm_status pm_compute_query_radii(pm_map* map, const pm_query_desc* desc, const float* d_qpos4, uint32_t nq,
                                 float* d_radii, void* stream);

/* ---- Batches of photon maps (no counterpart in the reference, which builds
 * and gathers one map per call).  Many maps of uneven size are built by one
 * sort and one tree, and queried by one persistent launch over a work queue
 * of all maps' queries; pm_batch_capture records both in a CUDA graph.
 *   Photons of map i: elements [photon_offsets[i], photon_offsets[i+1]) of
 *   d_pos4 / d_pow4 (host array of num_maps + 1 entries, starting at 0).
 *   Queries of map i: elements [query_offsets[i], query_offsets[i+1]) of
 *   d_qpos4 / d_qnrm4, answered with descs[i] (exact mode; k, r_max, filter,
 *   min_found per map).  d_rad4, d_r2, d_count are indexed like the queries;
 *   the neighbour rows of map i (k_i entries each, photon indices local to
 *   map i) start at entry sum_{j<i} q_j k_j of d_nbr.
 * Results are identical, bit for bit, to building and querying every map on
 * its own with pm_build / pm_query.  At most 65,536 maps and 2^31 - 1
 * photons per batch.  Batch queries always use one query per warp. */
typedef struct pm_batch pm_batch;
PM_API pm_status pm_batch_create(pm_batch** out);
PM_API pm_status pm_batch_destroy(pm_batch* batch);
/* Photons per leaf, warps per query block, query rounds per work chunk, and
 * whether the query traverses the 32-wide tree (wide != 0) or the binary one. */
PM_API pm_status pm_batch_set_tuning(pm_batch* batch, uint32_t leaf_size, int warps_per_block, int rounds_per_chunk,
                                     int wide);
PM_API pm_status pm_batch_build(pm_batch* batch, const float* d_pos4, const float* d_pow4,
                                const uint32_t* photon_offsets, uint32_t num_maps, int format, void* stream);
PM_API pm_status pm_batch_query(pm_batch* batch, const pm_query_desc* descs, const float* d_qpos4,
                                const float* d_qnrm4, const uint32_t* query_offsets, float* d_rad4, uint32_t* d_nbr,
                                float* d_r2, uint32_t* d_count, void* stream);
/* Records build + query with these arguments into a CUDA graph kept by the
 * handle (tables are uploaded and storage sized first; synchronous).
 * pm_batch_launch replays it on any stream: the graph reads the same device
 * buffers each time, so new photon and query values in them are picked up. */
PM_API pm_status pm_batch_capture(pm_batch* batch, const float* d_pos4, const float* d_pow4,
                                  const uint32_t* photon_offsets, uint32_t num_maps, int format,
                                  const pm_query_desc* descs, const float* d_qpos4, const float* d_qnrm4,
                                  const uint32_t* query_offsets, float* d_rad4, uint32_t* d_nbr, float* d_r2,
                                  uint32_t* d_count);
PM_API pm_status pm_batch_launch(pm_batch* batch, void* stream);
PM_API pm_status pm_batch_get_info(pm_batch* batch, pm_map_info* info, void* stream);
PM_API const char* pm_batch_last_error(const pm_batch* batch);
/* Times batch build + query over a grid of leaf sizes, warps per block,
 * rounds per chunk and tree width, applies the fastest, writes it to *best and leaves the
 * batch built with it.  Synchronous. */
PM_API pm_status pm_batch_autotune(pm_batch* batch, const float* d_pos4, const float* d_pow4,
                                   const uint32_t* photon_offsets, uint32_t num_maps, int format,
                                   const pm_query_desc* descs, const float* d_qpos4, const float* d_qnrm4,
                                   const uint32_t* query_offsets, float* d_rad4, pm_tuning* best, void* stream);

/* Phase timing with CUDA events recorded on the call's stream (off by
 * default).  pm_last_timings waits for the last recorded events. */
typedef struct pm_timings {
    float build_ms;          /* whole pm_build */
    float build_sort_ms;     /* Morton codes + radix sort inside pm_build */
    float query_ms;          /* whole pm_query */
    float query_sort_ms;     /* query Hilbert sort inside pm_query (0 when AS_GIVEN) */
    float query_kernel_ms;   /* the kNN kernel alone */
    uint32_t build_launches; /* kernels launched by the last pm_build */
    uint32_t query_launches; /* kernels launched by the last pm_query */
} pm_timings;
PM_API pm_status pm_set_profiling(pm_map* map, int enable);
PM_API pm_status pm_last_timings(pm_map* map, pm_timings* out);

/* Traversal counters of the last pm_query with a binary layout (PM_KBUF_HEAP or
 * PM_KBUF_GROUP; the 32-wide layout keeps no counters), collected
 * when profiling is enabled with level 2 (costs some speed).  Synchronous.
 * out[0..7]: queries, internal nodes visited (per warp), leaves visited (per
 * warp), photons tested (per warp), candidates appended, selections, radius
 * redos, queries started without a radius bound. */
PM_API pm_status pm_query_stats(pm_map* map, uint64_t* out, uint32_t count);

/* Blocks until the stream is idle, then fills info (including device error bits). */
PM_API pm_status pm_get_info(pm_map* map, pm_map_info* info, void* stream);
PM_API pm_status pm_clear_errors(pm_map* map, void* stream);

/* Copies the tree for structural validation: nodes as 16 uint32 each
 * (child 0: lo xyz, hi xyz, ref, count; child 1: same), and the photons in
 * tree order (pos4 with w = caller index bits, pow4 with w = direction bits).
 * Synchronous.  Any output pointer may be NULL. */
PM_API pm_status pm_export_tree(pm_map* map, uint32_t* host_nodes, uint32_t max_nodes, float* host_pos4,
                         float* host_pow4, uint32_t max_photons);

PM_API const char* pm_last_error(const pm_map* map);
PM_API const char* pm_status_string(pm_status s);
PM_API int pm_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PMGPU_H */
