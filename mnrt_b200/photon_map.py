"""Host-side mirror of MNRT's PhotonMap / KDTreePoint interface over the C ABI.

    pm = PhotonMap(max_photons, scene_min, scene_max, global_q_radius_max)
    pm.merge(photon_data, d_is_valid)        # PhotonMap::Merge       (PhotonMap.cpp:181)
    pm.scale_flux(1.0 / n_paths)             # PhotonMap::ScaleFlux   (PhotonMap.cpp:186)
    pm.build_map()                           # PhotonMap::BuildMap    (PhotonMap.cpp:157)
    pm.set_knn_target_count(100)             # PhotonMap::SetKNNTargetCount (PhotonMap.h:257)
    pm.gather_for(sp, rays, clr, idx, rad, recip)   # PhotonMap::GatherFor (PhotonMap.cpp:234)

plus the engine's direct calls (build / query / query_backward) on torch CUDA
tensors.  Device memory and streams come from torch; all computation runs in
libpmgpu.so.  Tensors are float32, contiguous, 4 floats per element.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _lib as L


def _ptr(t) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("engine buffers must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("engine buffers must be contiguous")
    return t.data_ptr()


def _stream(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


@dataclass
class PhotonData:
    """MNRT's PhotonData (KernelDefs.h:537-629): positions (xyz, azimuth phi)
    and powers (rgb, polar theta), or the engine's packed layout."""
    positions: torch.Tensor   # (n, 4) float32, CUDA
    powers: torch.Tensor      # (n, 4) float32, CUDA
    packed: bool = False

    @property
    def num_photons(self) -> int:
        return int(self.positions.shape[0])


@dataclass
class ShadingPoints:
    """Query side of MNRT's ShadingPoints (KernelDefs.h:160-291)."""
    pt_inter: torch.Tensor    # (n, 4) hit positions
    normals_s: torch.Tensor   # (n, 4) shading normals


@dataclass
class RayChunk:
    """The gather rays that produced the shading points (RayPool.h:162-178)."""
    origins: torch.Tensor     # (n, 4)
    dirs: torch.Tensor        # (n, 4)
    influences: torch.Tensor  # (n, 4)


class PhotonMap:
    def __init__(self, max_photons: int, scene_aabb_min=(0.0, 0.0, 0.0), scene_aabb_max=(1.0, 1.0, 1.0),
                 global_q_radius_max: float = 0.1, knn_target_count: int = 100):
        self._lib = L.load()
        h = C.c_void_p()
        lo = (C.c_float * 3)(*scene_aabb_min)
        hi = (C.c_float * 3)(*scene_aabb_max)
        st = self._lib.pm_create(C.byref(h), int(max_photons), lo, hi, float(global_q_radius_max))
        if st != L.PM_OK:
            raise L.PMError(st, "pm_create failed")
        self._h = h
        self.max_photons = int(max_photons)
        self.r_max = float(global_q_radius_max)
        self.k = int(knn_target_count)   # MNRT PhotonMap default m_knnTargetCount = 100 (PhotonMap.cpp:111)
        self._staged: list[PhotonData] = []
        self._num_staged = 0
        self.num_photons = 0

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- reference-shaped API ------------------------------------------------
    def set_knn_target_count(self, k: int) -> None:
        self.k = int(k)

    def get_photon_count(self) -> int:
        return self.num_photons

    def set_tuning(self, leaf_size: int = 32, warps_per_block: int = 4, rounds_per_chunk: int = 8,
                   queries_per_warp: int = 1, kbuf_layout: int = L.PM_KBUF_WIDE) -> None:
        L.check(self._lib.pm_set_tuning(self._h, leaf_size, warps_per_block, rounds_per_chunk, queries_per_warp,
                                        kbuf_layout), self._h)

    def autotune(self, positions: torch.Tensor, powers: torch.Tensor, qpos: torch.Tensor, qnrm: torch.Tensor,
                 max_sample: int = 0, packed: bool = True, stream=None, **kw) -> L.Tuning:
        """Picks leaf size, warps per block, rounds per chunk, queries per warp
        and k-buffer layout by timing build + query on a sample of the queries;
        the map is left built with the choice."""
        d = self.desc(**kw)
        best = L.Tuning()
        n = int(positions.shape[0])
        fmt = L.PM_PHOTONS_PACKED if packed else L.PM_PHOTONS_REFERENCE
        L.check(self._lib.pm_autotune(self._h, _ptr(positions), _ptr(powers), n, fmt, C.byref(d), _ptr(qpos),
                                      _ptr(qnrm), int(qpos.shape[0]), int(max_sample), C.byref(best),
                                      _stream(stream)), self._h)
        self.num_photons = n
        return best

    def reserve(self, max_photons: int, max_queries: int) -> None:
        L.check(self._lib.pm_reserve(self._h, int(max_photons), int(max_queries)), self._h)

    # -- engine API --------------------------------------------------------------
    def build(self, positions: torch.Tensor, powers: torch.Tensor, packed: bool = True, stream=None) -> None:
        n = int(positions.shape[0])
        if positions.dtype != torch.float32 or powers.dtype != torch.float32:
            raise ValueError("photon arrays must be float32")
        if positions.shape != (n, 4) or powers.shape != (n, 4):
            raise ValueError("photon arrays must be (n, 4)")
        fmt = L.PM_PHOTONS_PACKED if packed else L.PM_PHOTONS_REFERENCE
        L.check(self._lib.pm_build(self._h, _ptr(positions) if n else None, _ptr(powers) if n else None, n, fmt,
                                   _stream(stream)), self._h)
        self.num_photons = n

    def build_query_host(self, positions: torch.Tensor, powers: torch.Tensor, qpos: torch.Tensor, qnrm: torch.Tensor,
                         out: torch.Tensor | None = None, chunks: int = 1, packed: bool = True, stream=None,
                         **kw) -> torch.Tensor:
        """Build + query from host tensors (pinned for overlapped copies):
        photons in and build while the queries copy in, query, radiance out;
        chunks > 1 pipelines query pieces (pm_build_query_host).  Returns the
        host radiance (nq, 4); complete once the stream reaches this call."""
        for a in (positions, powers, qpos, qnrm):
            if a.is_cuda or a.dtype != torch.float32 or not a.is_contiguous() or a.dim() != 2 or a.shape[1] != 4:
                raise ValueError("host arrays must be contiguous float32 (n, 4) CPU tensors")
        n, nq = int(positions.shape[0]), int(qpos.shape[0])
        if out is None:
            out = torch.empty((nq, 4), dtype=torch.float32, pin_memory=True)
        d = self.desc(**kw)
        fmt = L.PM_PHOTONS_PACKED if packed else L.PM_PHOTONS_REFERENCE
        hp = lambda t: t.data_ptr() if t.numel() else None
        L.check(self._lib.pm_build_query_host(self._h, hp(positions), hp(powers), n, fmt, C.byref(d), hp(qpos),
                                              hp(qnrm), nq, hp(out), int(chunks), _stream(stream)), self._h)
        self.num_photons = n
        return out

    def desc(self, k=None, r_max=None, filter="box", cone_k=1.0, min_found=0, sorted_queries=True,
             mode=L.PM_MODE_EXACT, refine_iters=2) -> L.QueryDesc:
        return L.QueryDesc(k=int(k if k is not None else self.k), r_max=float(r_max if r_max is not None else self.r_max),
                           filter=L.FILTERS[filter] if isinstance(filter, str) else int(filter), cone_k=float(cone_k),
                           mode=int(mode), min_found=int(min_found),
                           order=L.PM_ORDER_SORTED if sorted_queries else L.PM_ORDER_AS_GIVEN,
                           refine_iters=int(refine_iters))

    def query(self, qpos: torch.Tensor, qnrm: torch.Tensor, want_nbr: bool = False, brute_force: bool = False,
              out: dict | None = None, stream=None, **kw) -> dict:
        """Exact-kNN radiance estimate; returns rad (nq,4) [, nbr (nq,k), r2, count]."""
        d = self.desc(**kw)
        nq = int(qpos.shape[0])
        dev = qpos.device
        if out is None:
            out = {"rad": torch.empty((nq, 4), dtype=torch.float32, device=dev),
                   "r2": torch.empty((nq,), dtype=torch.float32, device=dev),
                   "count": torch.empty((nq,), dtype=torch.int32, device=dev)}
            if want_nbr:
                out["nbr"] = torch.empty((nq, d.k), dtype=torch.int32, device=dev)
        fn = self._lib.pm_query_bruteforce if brute_force else self._lib.pm_query
        L.check(fn(self._h, C.byref(d), _ptr(qpos), _ptr(qnrm), nq, _ptr(out["rad"]), _ptr(out.get("nbr")),
                   _ptr(out.get("r2")), _ptr(out.get("count")), _stream(stream)), self._h)
        return out

    def info(self, stream=None) -> L.MapInfo:
        i = L.MapInfo()
        L.check(self._lib.pm_get_info(self._h, C.byref(i), _stream(stream)), self._h)
        return i

    def set_profiling(self, enable: int = 1) -> None:
        """1: phase timings with CUDA events; 2: also traversal counters."""
        L.check(self._lib.pm_set_profiling(self._h, int(enable)), self._h)

    STAT_NAMES = ("queries", "nodes_per_warp", "leaves_per_warp", "photons_per_warp", "candidates", "selections",
                  "redos", "unbounded")

    def query_stats(self) -> dict:
        """Traversal counters of the last query with a binary layout (needs set_profiling(2))."""
        import numpy as np
        out = np.zeros(8, np.uint64)
        L.check(self._lib.pm_query_stats(self._h, out.ctypes.data, 8), self._h)
        return dict(zip(self.STAT_NAMES, (int(x) for x in out)))

    def last_timings(self) -> L.Timings:
        t = L.Timings()
        L.check(self._lib.pm_last_timings(self._h, C.byref(t)), self._h)
        return t

    def clear_errors(self, stream=None) -> None:
        L.check(self._lib.pm_clear_errors(self._h, _stream(stream)), self._h)

    def export_tree(self):
        """(nodes uint32 (m+1, 16), pos float32 (n, 4), pow float32 (n, 4)) in tree order."""
        import numpy as np
        info = self.info()
        m = info.num_nodes + 1
        nodes = np.zeros((m, 16), np.uint32)
        pos = np.zeros((max(self.num_photons, 1), 4), np.float32)
        pw = np.zeros((max(self.num_photons, 1), 4), np.float32)
        L.check(self._lib.pm_export_tree(self._h, nodes.ctypes.data, m, pos.ctypes.data, pw.ctypes.data,
                                         pos.shape[0]), self._h)
        return nodes, pos[: self.num_photons], pw[: self.num_photons]

    def scale_flux(self, scale: float, stream=None) -> None:
        """PhotonMap::ScaleFlux (PhotonMap.cpp:186-193): RGB flux of the photons
        held (merged and built), direction bits untouched."""
        n = C.c_uint32(0)
        L.check(self._lib.pm_merged_count(self._h, C.byref(n)), self._h)
        if self.num_photons == 0 and n.value == 0:
            return
        L.check(self._lib.pm_scale_flux(self._h, float(scale), _stream(stream)), self._h)

    def query_backward(self, qpos: torch.Tensor, qnrm: torch.Tensor, grad_rad: torch.Tensor, nbr=None, count=None,
                       grad_pow: torch.Tensor | None = None, grad_pos: torch.Tensor | None = None, stream=None,
                       want_pow: bool = True, want_pos: bool = True, **kw):
        """Adjoint of query(): dL/dpower and dL/dposition (n, 4) in caller order.
        nbr / count: the forward's outputs (None recomputes the kNN)."""
        d = self.desc(**kw)
        nq = int(qpos.shape[0])
        dev = qpos.device
        n = max(self.num_photons, 1)
        if want_pow and grad_pow is None:
            grad_pow = torch.empty((n, 4), dtype=torch.float32, device=dev)
        if want_pos and grad_pos is None:
            grad_pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
        grad_rad = grad_rad.contiguous()
        if grad_rad.shape[1] != 4:
            g4 = torch.zeros((nq, 4), dtype=torch.float32, device=dev)
            g4[:, :3] = grad_rad
            grad_rad = g4
        L.check(self._lib.pm_query_backward(self._h, C.byref(d), _ptr(qpos), _ptr(qnrm), nq, _ptr(grad_rad),
                                            _ptr(nbr), None, _ptr(count), _ptr(grad_pow) if want_pow else None,
                                            _ptr(grad_pos) if want_pos else None, _stream(stream)), self._h)
        return grad_pow, grad_pos

    def set_backward_chunk(self, max_queries: int) -> None:
        L.check(self._lib.pm_set_backward_chunk(self._h, int(max_queries)), self._h)

    # -- reference build entry points ------------------------------------------------
    def merge(self, other: PhotonData, d_is_valid: torch.Tensor | None = None, stream=None) -> int:
        """PhotonMap::Merge (PhotonMap.cpp:181): appends the photons of other
        whose d_is_valid flag is non-zero (all when None); returns the count."""
        n = other.num_photons
        merged = C.c_uint32(0)
        L.check(self._lib.pm_merge(self._h, _ptr(other.positions) if n else None, _ptr(other.powers) if n else None,
                                   _ptr(d_is_valid), n, C.byref(merged), _stream(stream)), self._h)
        self._packed = other.packed
        return int(merged.value)

    def build_map(self, stream=None) -> bool:
        """PhotonMap::BuildMap (PhotonMap.cpp:157): the tree over the merged photons."""
        fmt = L.PM_PHOTONS_PACKED if getattr(self, "_packed", False) else L.PM_PHOTONS_REFERENCE
        L.check(self._lib.pm_build_merged(self._h, fmt, _stream(stream)), self._h)
        n = C.c_uint32(0)
        L.check(self._lib.pm_merged_count(self._h, C.byref(n)), self._h)
        self.num_photons = int(n.value)
        if getattr(self, "_icut", None) is not None and self.num_photons > 0:
            self.icut_build(stream=stream, **self._icut)   # PhotonMap.cpp:166-168
        return True

    def clear(self) -> None:
        """PhotonData::Clear: drops the merged photons."""
        L.check(self._lib.pm_clear_merged(self._h), self._h)

    # -- reference gather entry points ------------------------------------------------
    def gather_for(self, sp: ShadingPoints, rays: RayChunk, clr_diff_hit: torch.Tensor | None,
                   idx_shading_pts: torch.Tensor | None, io_radiance: torch.Tensor,
                   io_recip_dist: torch.Tensor | None = None, stream=None, **kw) -> None:
        """PhotonMap::GatherFor (PhotonMap.cpp:234-270): estimate at the gather
        hits (normal flipped toward the incoming ray) and accumulate
        clr.w * clr.rgb / pi * E * influence into io_radiance[idx] (and
        rsqrt(|hit - origin|^2) into io_recip_dist[idx]).  Defaults follow the
        reference: k = the map's kNN target count, R = its global radius,
        box filter, estimates from fewer than 8 photons zeroed."""
        kw.setdefault("filter", "box")
        kw.setdefault("min_found", 8)
        if getattr(self, "_icut", None) is not None:
            kw.setdefault("mode", L.PM_MODE_ICUT)   # GatherFor with illumination cuts (PhotonMap.cpp:244-257)
        d = self.desc(**kw)
        n = int(sp.pt_inter.shape[0])
        L.check(self._lib.pm_gather_for(self._h, C.byref(d), _ptr(sp.pt_inter), _ptr(sp.normals_s), _ptr(rays.dirs),
                                        _ptr(rays.origins), _ptr(rays.influences), _ptr(clr_diff_hit),
                                        _ptr(idx_shading_pts), n, _ptr(io_radiance), _ptr(io_recip_dist),
                                        _stream(stream)), self._h)

    def gather(self, sp: ShadingPoints, rays: RayChunk, clr_diff_hit: torch.Tensor, io_radiance: torch.Tensor,
               stream=None, **kw) -> None:
        """PhotonMap::Gather (PhotonMap.cpp:195-232): GatherFor with the
        shading points themselves as targets and no distance accumulator.
        Never uses illumination cuts (the reference disables them here,
        PhotonMap.cpp:206-224)."""
        kw.setdefault("mode", L.PM_MODE_EXACT)
        self.gather_for(sp, rays, clr_diff_hit, None, io_radiance, None, stream=stream, **kw)

    def visualize(self, sp: ShadingPoints, rays: RayChunk, io_radiance: torch.Tensor, stream=None) -> None:
        """PhotonMap::Visualize (PhotonMap.cpp:272-285): the nearest photon
        within 5 % of the global radius, white, no photon-count rule."""
        self.gather_for(sp, rays, None, None, io_radiance, None, stream=stream, k=1, r_max=0.05 * self.r_max,
                        min_found=0, mode=L.PM_MODE_EXACT)

    def compute_query_radii(self, qpos: torch.Tensor, out: torch.Tensor | None = None, stream=None,
                            **kw) -> torch.Tensor:
        """KDTreePoint::ComputeQueryRadii (KDTreePoint.cpp:229-248): the
        reference's histogram-refined query radius per point (ZHOU_COMPAT)."""
        kw.setdefault("mode", L.PM_MODE_ZHOU_COMPAT)
        d = self.desc(**kw)
        nq = int(qpos.shape[0])
        if out is None:
            out = torch.empty((nq,), dtype=torch.float32, device=qpos.device)
        L.check(self._lib.pm_compute_query_radii(self._h, C.byref(d), _ptr(qpos), nq, _ptr(out), _stream(stream)),
                self._h)
        return out

    # -- illumination cuts (PhotonMap.cpp:287-452, GPU/illumcut.cu) -------------------
    def set_illum_cuts(self, enabled: bool = True, use_leafs: bool = True, level_emin: int = 12,
                       refine_iters: int = 4, accuracy: float = 0.2, **node_query) -> None:
        """MNRTSettings::SetUseIllumCuts and the ICut* settings (defaults as
        MNRTSettings.h:491-523): build_map then builds the cut and gather_for
        with idx_shading_pts interpolates it, as the reference's GatherFor."""
        self._icut = (dict(use_leafs=use_leafs, level_emin=level_emin, refine_iters=refine_iters, accuracy=accuracy,
                           **node_query) if enabled else None)

    def icut_build(self, use_leafs: bool = True, level_emin: int = 12, refine_iters: int = 4,
                   accuracy: float = 0.2, node_normals: torch.Tensor | None = None, stream=None, **kw) -> None:
        """Builds the illumination cut of the current tree.  kw describes the
        node-centre estimate (k, r_max, filter, min_found, mode); defaults are
        the reference's: the map's k and R, box filter, 8 photons at least."""
        kw.setdefault("filter", "box")
        kw.setdefault("min_found", 8)
        d = self.desc(**kw)
        c = L.IcutDesc(int(bool(use_leafs)), int(level_emin), int(refine_iters), float(accuracy))
        L.check(self._lib.pm_icut_build(self._h, C.byref(c), C.byref(d), _ptr(node_normals), _stream(stream)),
                self._h)

    def icut_slot_count(self) -> int:
        n = C.c_uint32(0)
        L.check(self._lib.pm_icut_slot_count(self._h, C.byref(n)), self._h)
        return int(n.value)

    def icut_node_centers(self, device="cuda", stream=None) -> torch.Tensor:
        """(slots, 4): box centre xyz and largest box side per slot."""
        out = torch.empty((self.icut_slot_count(), 4), dtype=torch.float32, device=device)
        L.check(self._lib.pm_icut_node_centers(self._h, _ptr(out), _stream(stream)), self._h)
        return out

    def icut_interpolate(self, qpos: torch.Tensor, qnrm: torch.Tensor, r_max: float | None = None,
                         stream=None) -> torch.Tensor:
        nq = int(qpos.shape[0])
        out = torch.empty((nq, 4), dtype=torch.float32, device=qpos.device)
        r = self.r_max if r_max is None else r_max
        L.check(self._lib.pm_icut_interpolate(self._h, float(r), _ptr(qpos), _ptr(qnrm), nq, _ptr(out),
                                              _stream(stream)), self._h)
        return out

    def icut_export(self) -> dict:
        """Host copies of the cut: coarse, final, level, center, normal, est, exact."""
        import numpy as np
        ns = self.icut_slot_count()
        u = {k: np.empty(ns, np.uint32) for k in ("coarse", "final", "level")}
        f = {k: np.empty((ns, 4), np.float32) for k in ("center", "normal", "est", "exact")}
        L.check(self._lib.pm_icut_export(self._h, ns, *(u[k].ctypes.data for k in ("coarse", "final", "level")),
                                         *(f[k].ctypes.data for k in ("center", "normal", "est", "exact"))), self._h)
        return {**u, **f}
