#!/usr/bin/env python
"""Benchmark: photon-map kd-tree build + exact-kNN radiance estimate on B200.

One step = one pass of the hot path over one synthetic photon map: build the
point kd-tree over N photons, then the k-nearest radiance estimate at Q query
points (Hilbert-order query sort included).  Default workload ("plain"): 1,048,576 photons
(80% uniform on the five room walls, 20% in a sigma=0.01 caustic on the
floor), 2,073,600 uniform wall queries (one per 1920x1080 pixel), k = 100,
R = 0.05, cone filter, FP32.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (one rank per GPU) the plain and final-gather workloads build
the same map on every rank and divide its queries into contiguous ranges
(mnrt_b200/shard.py query_range; no data exchange, the radiance stays on the
rank that computed it): scaling is strong and value is all queries over the
slowest rank's step.  --division replicas instead gives every rank its own
seeded map and query set (weak scaling); the icut workload always runs
replicas.  The batch workload divides its maps over the ranks by LPT; the
diff workload builds the map on every rank, divides the queries and sums the
adjoint's partial gradients with one all-reduce (mnrt_b200/shard.py).
--impl reference times the CPU port of the reference algorithm (oracle/,
multithreaded kd-tree) on the same workload.

The default run (plain workload, one GPU) adds three sub-objects measured
after its own timed region, in the same process: "final_gather" (4,194,304
photons, 8,388,608 queries, k = 64: Hilbert-sorted against as-given query
order), "batch" (64 maps in one CUDA graph against 64 sequential per-map
calls) and "diff" (forward and forward + adjoint times, gradient descent on
the powers).  --no-extras skips them.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "kNN radiance estimates/s (kd-tree build + k-nearest query per step)"
UNIT = "queries/s"


def workload_config(name: str) -> dict:
    from mnrt_b200 import gen
    c = dict(gen.CONFIGS[name])
    desc = (f"{name}: {c['n']:,} photons ({int(100 * (1 - c.get('caustic_frac', 0)))}% walls / "
            f"{int(100 * c.get('caustic_frac', 0))}% caustic), {c['nq']:,} wall queries"
            f"{' (50% clustered)' if c.get('cluster_frac') else ''}, k={c['k']}, R={c['r_max']}, "
            f"{c['filter']} filter, FP32")
    c["workload"] = desc
    return c


def make_inputs(cfg: dict, rank: int):
    from mnrt_b200 import gen
    ph = gen.photons(cfg["n"], seed=1000 + rank, caustic_frac=cfg.get("caustic_frac", 0.2),
                     power_mean=cfg.get("power_mean"))
    q = gen.queries(cfg["nq"], seed=2000 + rank, cluster_frac=cfg.get("cluster_frac", 0.0))
    return ph, q


# ------------------------------------------------------------- CPU legs --

def cpu_reference_step(ph, q, cfg, sample: int, threads: int, rng: np.random.Generator):
    """One CPU step: full kd-tree build (multithreaded) + a bounded query
    sample, scaled to Q."""
    from oracle import oracle
    t0 = time.perf_counter()
    tree = oracle.KdTree(ph.pos, threads=threads)
    t1 = time.perf_counter()
    sel = rng.choice(q.n, size=min(sample, q.n), replace=False)
    qp, qn = q.pos[sel], q.nrm[sel]
    idx, _d2, cnt, _r2 = tree.knn(qp, cfg["k"], cfg["r_max"], threads=threads)
    oracle.radiance_fp64(ph.pos, ph.pow, qp, qn, idx, cnt, cfg["k"], cfg["r_max"], cfg["filter"], 1.0, 0,
                         threads=threads)
    t2 = time.perf_counter()
    step_s = (t1 - t0) + (t2 - t1) * q.n / len(sel)
    return q.n / step_s, t1 - t0, (t2 - t1) / len(sel)


def calibrate_sample(ph, q, cfg, threads: int, target_s: float) -> int:
    from oracle import oracle
    tree = oracle.KdTree(ph.pos)
    probe = min(20000, q.n)
    t0 = time.perf_counter()
    tree.knn(q.pos[:probe], cfg["k"], cfg["r_max"], threads=threads)
    per = (time.perf_counter() - t0) / probe
    return int(max(1000, min(q.n, target_s / max(per, 1e-9))))


def run_reference(args, cfg) -> dict:
    from oracle import oracle
    ph, q = make_inputs(cfg, 0)
    threads = oracle.threads_available()
    sample = calibrate_sample(ph, q, cfg, threads, target_s=1.5)
    rng = np.random.default_rng(7)
    for _ in range(args.warmup):
        cpu_reference_step(ph, q, cfg, sample, threads, rng)
    vals, builds = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, b, _per = cpu_reference_step(ph, q, cfg, sample, threads, rng)
        vals.append(v)
        builds.append(b)
    wall = time.perf_counter() - t0
    tb = time.perf_counter()
    oracle.KdTree(ph.pos, threads=1)   # the build on one thread, for the record
    build_1t_ms = 1000.0 * (time.perf_counter() - tb)
    value = float(np.mean(vals))
    sample_desc = (f"kd-tree build over all {cfg['n']:,} photons ({threads} threads) + {sample:,} of {cfg['nq']:,} "
                   f"queries per step (random subset), query time scaled to all queries")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * cfg["nq"] / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "photons": cfg["n"], "queries": cfg["nq"], "k": cfg["k"],
                   "r_max": cfg["r_max"], "filter": cfg["filter"], "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample_desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "build_ms_cpu": 1000.0 * float(np.mean(builds)), "build_ms_cpu_threads": threads,
        "build_ms_cpu_1_thread": build_1t_ms, "wall_s": wall,
        "note": "the reference ships no CPU path and cannot be built here; this is the oracle's port of its "
                "algorithm (exact kNN, multithreaded kd-tree)",
    }


# ------------------------------------------------------------------ GPU --

class ClockSampler:
    """Clock and throttle samples while the timed region runs: NVML every
    5 ms from a thread, plus the nvidia-smi line of the profiling recipe every
    200 ms.  The GPU is found by the CUDA device's PCI bus id."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.file = None
        self.nvml = None
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = None
        self._thread = None

    def _bus_id(self) -> str | None:
        try:
            import torch
            p = torch.cuda.get_device_properties(self.idx)
            return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            return None

    def __enter__(self):
        import threading
        bus = self._bus_id()
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByPciBusId(bus) if bus else nv.nvmlDeviceGetHandleByIndex(self.idx)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = (nv, h)
            self._stop = threading.Event()

            def loop():
                while not self._stop.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        pass
                    self._stop.wait(0.005)

            self._thread = threading.Thread(target=loop, daemon=True)
            self._thread.start()
        except Exception:
            self.nvml = None
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", bus if bus else str(self.idx),
                                          f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.proc is not None and self.file is not None:
            self.file.flush()
            for line in Path(self.file.name).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.file.name)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"}
        reasons |= {n for mhz, bits in self.samples for b, n in self.REASONS.items() if bits & b}
        sm = [m for m, _ in self.samples] or [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = self.max_mhz or max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(np.min(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(self.samples), "smi_samples": len(rows),
                "source": "NVML every 5 ms + nvidia-smi every 200 ms"}


def rank_max(values: list[float], dev=None) -> list[float]:
    """Max over ranks of each value (device times of the timed region); the
    values themselves without a process group of more than one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel: str, workload: str, field: str = "dram_bytes_per_launch"):
    """Bytes per launch (DRAM by default) from the committed ncu summary, if one exists."""
    f = ROOT / "profiles" / f"{kernel}_{workload}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(field + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def init_ranks():
    """(world, rank, local rank, device) from the torchrun environment; a
    world above one gets an NCCL process group with a short timeout."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    return world, rank, local, dev


def close_ranks(world: int) -> None:
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def barrier(world: int) -> None:
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()


def run_ours(args, cfg, light: bool = False) -> dict | None:
    """The plain one-map step.  light: the device-resident step only (no
    end-to-end leg, no build median, no CPU baseline): the form the default
    run uses for its final-gather sub-measurement."""
    import torch
    import torch.distributed as dist

    world, rank, local, dev = init_ranks()

    from mnrt_b200 import gen
    from mnrt_b200.photon_map import PhotonMap
    from mnrt_b200.shard import query_range

    # N > 1: one map, its queries divided into contiguous ranges (every rank
    # builds the same map); --division replicas gives every rank its own map
    division = args.division or ("queries" if world > 1 else "replicas")
    if division == "queries":
        ph, q_all = make_inputs(cfg, 0)
        qa, qb = query_range(q_all.n, rank, world)
        q = gen.QuerySet(np.ascontiguousarray(q_all.pos[qa:qb]), np.ascontiguousarray(q_all.nrm[qa:qb]))
        Q_job = q_all.n
    else:
        ph, q = make_inputs(cfg, rank)
        Q_job = world * q.n
    N, Q, k, R = cfg["n"], q.n, cfg["k"], cfg["r_max"]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_pos, h_pow, h_qpos, h_qnrm = pin(ph.pos), pin(ph.pow), pin(q.pos), pin(q.nrm)
    h_rad = torch.empty((Q, 4), dtype=torch.float32).pin_memory()
    d_pos, d_pow = h_pos.to(dev), h_pow.to(dev)
    d_qpos, d_qnrm = h_qpos.to(dev), h_qnrm.to(dev)
    d_rad = torch.empty((Q, 4), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MiB > 126 MB L2

    pm = PhotonMap(N, global_q_radius_max=R, knn_target_count=k)
    tuning = "defaults"
    if args.leaf or args.wpb or args.rounds or args.qpw or args.layout >= 0:
        pm.set_tuning(leaf_size=args.leaf or 32, warps_per_block=args.wpb or 4, rounds_per_chunk=args.rounds or 8,
                      queries_per_warp=args.qpw or 1, kbuf_layout=args.layout if args.layout >= 0 else 2)
        tuning = "set by flags"
    elif not args.no_autotune:   # untimed: picks the kernel setting on a query sample
        t = pm.autotune(d_pos, d_pow, d_qpos, d_qnrm, max_sample=0, k=k, r_max=R, filter=cfg["filter"])
        tuning = {"leaf_size": t.leaf_size, "warps_per_block": t.warps_per_block,
                  "rounds_per_chunk": t.rounds_per_chunk, "queries_per_warp": t.queries_per_warp,
                  "kbuf_layout": t.kbuf_layout, "chosen_by": "pm_autotune over all queries"}
    pm.reserve(N, Q)
    pm.set_profiling(True)
    out = {"rad": d_rad}
    qkw = dict(k=k, r_max=R, filter=cfg["filter"], cone_k=1.0, sorted_queries=not args.unsorted)

    def step():
        pm.build(d_pos, d_pow)
        pm.query(d_qpos, d_qnrm, out=out, **qkw)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = pm.info().launches
    builds, queries, kernels, sorts, steps_ms = [], [], [], [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()                       # evict L2 between timed steps (not timed)
            e0.record()
            step()
            e1.record()
            e1.synchronize()
            steps_ms.append(e0.elapsed_time(e1))
            t = pm.last_timings()
            builds.append(t.build_ms)
            queries.append(t.query_ms)
            kernels.append(t.query_kernel_ms)
            sorts.append(t.query_sort_ms)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clk.summary()
    launches = pm.info().launches - launches0
    info = pm.info()
    total_ms = rank_max([float(np.sum(steps_ms))], dev)[0]
    ms_per_step = total_ms / args.steps
    value = Q_job / (ms_per_step / 1000.0)

    if light:
        kern_ms = float(np.mean(kernels))
        res = {"value": value, "ms_per_step": ms_per_step, "build_ms": float(np.mean(builds)),
               "query_sort_ms": float(np.mean(sorts)), "query_kernel_ms": kern_ms,
               "query_kernel_queries_per_s": Q / (kern_ms / 1000.0), "clocks": clocks,
               "device_errors": info.device_errors, "gpu_launches": int(launches), "tuning": tuning}
        pm.close()
        close_ranks(world)
        return res if rank == 0 else None

    # end to end through the public API: pinned host in, host radiance out.
    # pm_build_query_host copies the photons in and builds while the queries
    # copy in (one piece: measured fastest, see --chunks).
    e2e_ms = []
    hkw = {kk: v for kk, v in qkw.items()}
    for i in range(args.warmup + args.steps):
        flush.zero_()
        e0.record()
        pm.build_query_host(h_pos, h_pow, h_qpos, h_qnrm, out=h_rad, chunks=args.chunks, **hkw)
        e1.record()
        e1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_total = rank_max([float(np.sum(e2e_ms))], dev)[0]
    e2e_value = Q_job / (e2e_total / args.steps / 1000.0)
    if not torch.equal(h_rad.view(torch.int32), d_rad.cpu().view(torch.int32)):
        raise RuntimeError("host-buffer path and device path disagree")

    # the build alone: median of 20 warm builds (untimed by the step figure)
    build_alone = []
    for _ in range(20):
        pm.build(d_pos, d_pow)
        build_alone.append(pm.last_timings().build_ms)
    build_median_ms = rank_max([float(np.median(build_alone))], dev)[0]

    kern_ms = float(np.mean(kernels))
    nodes = info.num_nodes
    alg_bytes = 48 * Q + 32 * N + 64 * (nodes + 1)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kern_ms / 1000.0) / 1e9
    build_ms = float(np.mean(builds))
    build_bytes = 68 * N + 64 * (nodes + 1)
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if division == "queries" and world > 1 else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "photons": N, "queries": Q_job, "k": k, "r_max": R,
                   "filter": cfg["filter"], "query_order": "as given" if args.unsorted else "Hilbert-sorted",
                   "l2": "flushed between steps (256 MiB write, untimed)",
                   "parallelism": (f"one map built on each of {world} GPUs, its queries divided into {world} "
                                   f"contiguous ranges (rank 0: {Q:,}), no exchange"
                                   if division == "queries" and world > 1 else
                                   f"{world} independent replica(s), one per GPU"),
                   "tuning": tuning},
        "build_ms": build_ms, "build_ms_median_of_20_warm": build_median_ms, "query_ms": float(np.mean(queries)), "query_sort_ms": float(np.mean(sorts)),
        "query_kernel_ms": kern_ms, "query_only_mqueries_per_s": Q / (float(np.mean(queries)) / 1000.0) / 1e6,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profiled_traffic("k_knn_group", args.config), "kernel": "k_knn_group",
                     "l2_traffic": profiled_traffic("k_knn_group", args.config, "l2_bytes_per_launch"),
                     "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peak_kind},
        "roofline_build": {"bound": "hbm", "achieved": build_bytes / (build_ms / 1000.0) / 1e9, "peak": peak,
                           "unit": "GB/s", "frac": build_bytes / (build_ms / 1000.0) / 1e9 / peak,
                           "algorithmic_bytes": build_bytes},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 32 * N + 32 * Q,
                "per_rank_bytes": world > 1,
                "d2h_bytes_per_step": 16 * Q, "call": "pm_build_query_host (pinned host buffers)",
                "chunks": args.chunks, "ms_per_step": e2e_total / args.steps},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "tree_nodes": nodes,
        "device_errors": info.device_errors,
    }
    close_ranks(world)
    if rank != 0:
        return None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        threads = oracle.threads_available()
        sample = calibrate_sample(ph, q, cfg, threads, target_s=8.0)
        v, b, per = cpu_reference_step(ph, q, cfg, sample, threads, np.random.default_rng(11))
        result["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"kd-tree build over all {N:,} photons ({1000 * b:.0f} ms on {threads} threads) + {sample:,} "
                      f"random queries of {Q:,}, query time scaled to all queries"}
    return result


def run_diff(args, cfg) -> dict | None:
    """Differentiation workload: forward (build + query with neighbour lists)
    and adjoint (dL/dpower, dL/dposition) of L = sum |E - T|^2, T from powers
    scaled by seeded U[0.5, 1.5]; then gradient descent on the powers.
    Under torchrun the map is built on every rank and the queries are divided
    (contiguous ranges); each rank's adjoint is a partial sum over its
    queries, and one all-reduce of the two gradients (inside the timed step)
    completes it.  Loss and line-search sums are all-reduced scalars."""
    import torch
    from mnrt_b200.photon_map import PhotonMap
    from mnrt_b200.shard import allreduce_gradients, allreduce_scalars, query_range

    world, rank, local, dev = init_ranks()
    ph, q = make_inputs(cfg, 0)          # one map and one query set, divided by query range
    N, Q, k, R, filt = cfg["n"], cfg["nq"], cfg["k"], cfg["r_max"], cfg["filter"]
    qa, qb = query_range(Q, rank, world)
    Qr = qb - qa
    rng = np.random.default_rng(4242)
    tpow = ph.pow.copy()
    tpow[:, :3] *= rng.uniform(0.5, 1.5, size=(N, 3)).astype(np.float32)
    d_pos, d_pow = torch.from_numpy(ph.pos).to(dev), torch.from_numpy(ph.pow).to(dev)
    d_tpow = torch.from_numpy(tpow).to(dev)
    d_qpos = torch.from_numpy(np.ascontiguousarray(q.pos[qa:qb])).to(dev)
    d_qnrm = torch.from_numpy(np.ascontiguousarray(q.nrm[qa:qb])).to(dev)
    pm = PhotonMap(N, global_q_radius_max=R, knn_target_count=k)
    kw = dict(k=k, r_max=R, filter=filt)
    tuning = "defaults"
    if not args.no_autotune:   # untimed: the forward's kernel setting, as the plain workload picks it
        t = pm.autotune(d_pos, d_pow, d_qpos, d_qnrm, max_sample=0, **kw)
        tuning = {"leaf_size": t.leaf_size, "warps_per_block": t.warps_per_block,
                  "rounds_per_chunk": t.rounds_per_chunk, "queries_per_warp": t.queries_per_warp,
                  "kbuf_layout": t.kbuf_layout, "chosen_by": "pm_autotune over all queries"}
    pm.reserve(N, Qr)
    pm.build(d_pos, d_tpow)
    target = pm.query(d_qpos, d_qnrm, **kw)["rad"][:, :3].clone()
    out = {"rad": torch.empty((Qr, 4), dtype=torch.float32, device=dev),
           "nbr": torch.empty((Qr, k), dtype=torch.int32, device=dev),
           "count": torch.empty((Qr,), dtype=torch.int32, device=dev)}
    out_plain = {"rad": torch.empty((Qr, 4), dtype=torch.float32, device=dev)}
    g = torch.zeros((Qr, 4), dtype=torch.float32, device=dev)
    gpow = torch.empty((N, 4), dtype=torch.float32, device=dev)
    gpos = torch.empty((N, 4), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def fwd(o):
        pm.build(d_pos, d_pow)
        pm.query(d_qpos, d_qnrm, out=o, **kw)

    def bwd():
        g[:, :3] = 2.0 * (out["rad"][:, :3] - target)
        pm.query_backward(d_qpos, d_qnrm, g, nbr=out["nbr"], count=out["count"], grad_pow=gpow, grad_pos=gpos, **kw)
        allreduce_gradients(gpow, gpos)

    for _ in range(args.warmup):
        fwd(out_plain); fwd(out); bwd()
    t_fwd, t_bwd = [], []
    barrier(world)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            ev[0].record(); fwd(out_plain); ev[1].record(); ev[1].synchronize()
            flush.zero_()
            ev[0].record(); fwd(out); ev[2].record(); bwd(); ev[3].record(); ev[3].synchronize()
            t_fwd.append(ev[0].elapsed_time(ev[2]))
            t_bwd.append(ev[2].elapsed_time(ev[3]))
    clocks = clk.summary()
    # forward without neighbour lists, timed on its own
    plain = []
    for _ in range(args.steps):
        flush.zero_()
        ev[0].record(); fwd(out_plain); ev[1].record(); ev[1].synchronize()
        plain.append(ev[0].elapsed_time(ev[1]))
    barrier(world)
    fwd_ms, bwd_ms, plain_ms, step_ms = rank_max([float(np.mean(t_fwd)), float(np.mean(t_bwd)), float(np.mean(plain)),
                                                  float(np.mean(np.add(t_fwd, t_bwd)))], dev)

    # gradient descent on the powers; E is linear in them, so the step along
    # -dL/dpower is the exact line-search minimiser alpha = |grad|^2 / |A grad|^2
    steps = args.gd_steps
    losses = []
    pw = d_pow.clone()
    dirp = torch.zeros_like(pw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(steps + 1):
        pm.build(d_pos, pw)
        pm.query(d_qpos, d_qnrm, out=out, **kw)
        res = out["rad"][:, :3] - target
        losses.append(allreduce_scalars([float((res.double() ** 2).sum())])[0])
        if it == steps:
            break
        g[:, :3] = 2.0 * res
        pm.query_backward(d_qpos, d_qnrm, g, nbr=out["nbr"], count=out["count"], grad_pow=gpow, want_pos=False, **kw)
        allreduce_gradients(gpow)
        dirp[:, :3] = gpow[:, :3]
        dirp[:, 3] = pw[:, 3]                       # direction bits ride along
        pm.build(d_pos, dirp)
        ag = pm.query(d_qpos, d_qnrm, out=out_plain, **kw)["rad"][:, :3].double()
        num = float((gpow[:, :3].double() ** 2).sum())
        den = 2.0 * allreduce_scalars([float((ag ** 2).sum())])[0]
        alpha = num / den if den > 0 else 0.0
        pw[:, :3] -= float(alpha) * gpow[:, :3]
    torch.cuda.synchronize()
    gd_s = time.perf_counter() - t0
    pm.close()
    close_ranks(world)
    if rank != 0:
        return None
    return {
        "metric": "forward + adjoint time of the radiance estimate (differentiation workload)",
        "value": step_ms, "unit": "ms", "higher_is_better": False, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "scaling": "strong", "dtype": "f32 (adjoint sums in f64)", "data": "synthetic",
        "config": {"workload": cfg["workload"], "photons": N, "queries": Q, "k": k, "r_max": R, "filter": filt,
                   "l2": "flushed between steps (256 MiB write, untimed)",
                   "parallelism": "one GPU" if world == 1 else
                   f"map on every rank, queries divided over {world} ranks, gradient all-reduce (NCCL, f64)",
                   "tuning": tuning},
        "clocks": clocks,
        "forward_ms": fwd_ms, "forward_no_lists_ms": plain_ms, "backward_ms": bwd_ms,
        "fwd_bwd_over_fwd": (fwd_ms + bwd_ms) / fwd_ms, "fwd_bwd_over_fwd_no_lists": (fwd_ms + bwd_ms) / plain_ms,
        "gradient_descent": {"steps": steps, "loss_first": losses[0], "loss_last": losses[-1],
                             "loss_ratio": losses[-1] / losses[0] if losses[0] > 0 else None,
                             "seconds": gd_s, "line_search": "exact (E is linear in the powers)"},
    }


def run_icut(args, cfg) -> dict | None:
    """Final gathering with illumination cuts (the reference's default
    GatherFor, PhotonMap.cpp:244-257): per step, build the tree and its cut
    (leaves as the coarse cut, exact-kNN irradiance at every node centre,
    4 refinement rounds, accuracy 0.2), then interpolate the cut at every
    query.  Also times the photon-search estimate on the same queries.
    Under torchrun every rank runs its own map and queries (replicas)."""
    import torch
    from mnrt_b200.photon_map import PhotonMap

    world, rank, local, dev = init_ranks()
    ph, q = make_inputs(cfg, rank)
    N, Q, k, R = cfg["n"], cfg["nq"], cfg["k"], cfg["r_max"]
    d_pos, d_pow = torch.from_numpy(ph.pos).to(dev), torch.from_numpy(ph.pow).to(dev)
    d_qp, d_qn = torch.from_numpy(q.pos).to(dev), torch.from_numpy(q.nrm).to(dev)
    pm = PhotonMap(N, global_q_radius_max=R, knn_target_count=k)
    pm.reserve(N, Q)
    out = torch.empty((Q, 4), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    qdesc = dict(k=k, r_max=R, filter="box", min_found=8)

    def step():
        pm.build(d_pos, d_pow)
        ev[1].record()
        pm.icut_build(**qdesc)
        ev[2].record()
        pm._lib.pm_icut_interpolate(pm._h, float(R), d_qp.data_ptr(), d_qn.data_ptr(), Q, out.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream)

    for _ in range(args.warmup):
        step()
    tot, cut, interp = [], [], []
    barrier(world)
    for _ in range(args.steps):
        flush.zero_()
        ev[0].record(); step(); ev[3].record(); ev[3].synchronize()
        tot.append(ev[0].elapsed_time(ev[3]))
        cut.append(ev[1].elapsed_time(ev[2]))
        interp.append(ev[2].elapsed_time(ev[3]))
    # the photon-search estimate on the same queries, for comparison
    qo = {"rad": torch.empty((Q, 4), dtype=torch.float32, device=dev)}
    for _ in range(args.warmup):
        pm.query(d_qp, d_qn, out=qo, **qdesc)
    knn = []
    for _ in range(args.steps):
        flush.zero_()
        ev[0].record(); pm.query(d_qp, d_qn, out=qo, **qdesc); ev[1].record(); ev[1].synchronize()
        knn.append(ev[0].elapsed_time(ev[1]))
    barrier(world)
    ns = pm.icut_slot_count()
    cutx = pm.icut_export()
    info = pm.info()
    tot_ms, cut_ms, interp_ms, knn_ms = rank_max([float(np.mean(x)) for x in (tot, cut, interp, knn)], dev)
    irr = out[:, :3].sum(1).cpu().numpy()
    direct = qo["rad"][:, :3].sum(1).cpu().numpy()
    ok = direct > 0
    ratio = irr[ok] / direct[ok]
    res = {
        "metric": "final-gather irradiance from the illumination cut: queries/s (build + cut + interpolation per step)",
        "value": world * Q / (tot_ms / 1000.0), "unit": "queries/s", "higher_is_better": True, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "scaling": "weak", "dtype": "f32 (interpolation sums in f64)",
        "data": "synthetic",
        "config": {"workload": cfg["workload"] + "; illumination cut: leaves as coarse cut, 4 refinement rounds, "
                               "accuracy 0.2, node-centre estimate exact kNN (box, min_found 8)",
                   "photons": N, "queries": Q, "k": k, "r_max": R,
                   "l2": "flushed between steps (256 MiB write, untimed)",
                   "parallelism": f"{world} independent replica(s), one per GPU"},
        "step_ms": tot_ms, "build_ms": tot_ms - cut_ms - interp_ms, "cut_build_ms": cut_ms,
        "interpolation_ms": interp_ms, "interpolation_queries_per_s": Q / (interp_ms / 1000.0),
        "knn_query_ms": knn_ms, "interpolation_speedup_over_knn": knn_ms / interp_ms,
        "slots": ns, "cut_slots": int(cutx["final"].sum()), "device_errors": info.device_errors,
        "interp_over_knn_estimate": {"median": float(np.median(ratio)),
                                     "p25": float(np.percentile(ratio, 25)), "p75": float(np.percentile(ratio, 75))},
    }
    close_ranks(world)
    if rank != 0:
        pm.close()
        return None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        nodes, _tpos, _tpow = pm.export_tree()
        threads = oracle.threads_available()
        rng = np.random.default_rng(7)
        sample = min(Q, 200000)
        idx = rng.choice(Q, sample, replace=False)
        t0 = time.perf_counter()
        oracle.icut_interp(nodes, cutx["final"], cutx["center"], cutx["normal"], cutx["exact"], q.pos[idx],
                           q.nrm[idx], R, threads)
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": sample / dt, "unit": "queries/s", "cores": threads, "kind": "port",
                               "sample": f"the oracle's interpolation over the engine's cut, {sample:,} random "
                                         f"queries of {Q:,} (interpolation stage only)"}
    pm.close()
    return res


def run_batch(args) -> dict | None:
    """Config 3: 64 photon maps (photon counts log-uniform in [1e4, 2e6], query
    counts log-uniform in [1e3, 1e6], k from {16, 32, 64, 128}, R = 0.05),
    built and queried as one batch (eager and CUDA-graph replay) against 64
    sequential per-map build + query calls.  Under torchrun the maps are
    divided over the ranks by LPT over photons + queries; each rank builds and
    queries its own maps as one batch, with no exchange: the whole batch's
    queries over the slowest rank's time."""
    import torch
    from mnrt_b200 import gen
    from mnrt_b200.batch import PhotonMapBatch
    from mnrt_b200.photon_map import PhotonMap
    from mnrt_b200.shard import lpt_assign, map_costs

    world, rank, local, dev = init_ranks()
    spec = gen.batch_spec(args.maps, seed=777)
    N_all, Q_all = int(np.sum(spec.n)), int(np.sum(spec.nq))
    mine = lpt_assign(map_costs(spec.n, spec.nq), world)[rank]
    ns, nqs, ks = [int(spec.n[i]) for i in mine], [int(spec.nq[i]) for i in mine], [int(spec.k[i]) for i in mine]
    phs = [gen.photons(spec.n[i], seed=spec.seeds[i], caustic_frac=0.2) for i in mine]
    qs = [gen.queries(spec.nq[i], seed=spec.seeds[i] + 500) for i in mine]
    descs = [dict(k=k, r_max=0.05, filter="cone") for k in ks]
    poff = np.concatenate([[0], np.cumsum(ns)]).astype(np.uint32)
    qoff = np.concatenate([[0], np.cumsum(nqs)]).astype(np.uint32)
    N, Q = int(poff[-1]), int(qoff[-1])
    cat = lambda xs: torch.from_numpy(np.concatenate(xs) if xs else np.zeros((0, 4), np.float32)).to(dev)
    d_pos, d_pw = cat([p.pos for p in phs]), cat([p.pow for p in phs])
    d_qp, d_qn = cat([q.pos for q in qs]), cat([q.nrm for q in qs])
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    clock_runs = []

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        barrier(world)
        ts = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                flush.zero_()
                e0.record(); fn(); e1.record(); e1.synchronize()
                ts.append(e0.elapsed_time(e1))
        clock_runs.append(clk.summary())
        barrier(world)
        return float(np.mean(ts))

    # sequential plain-form calls, one per map (storage reserved beforehand)
    maps = []
    for i, (ph, q) in enumerate(zip(phs, qs)):
        pm = PhotonMap(ph.n, global_q_radius_max=0.05, knn_target_count=ks[i])
        pm.reserve(ph.n, q.n)
        a, b = int(poff[i]), int(poff[i + 1])
        c, d = int(qoff[i]), int(qoff[i + 1])
        out = {"rad": torch.empty((q.n, 4), dtype=torch.float32, device=dev)}
        maps.append((pm, d_pos[a:b], d_pw[a:b], d_qp[c:d], d_qn[c:d], out, descs[i]))

    def sequential():
        for pm, p, w, qp, qn, out, dsc in maps:
            pm.build(p, w)
            pm.query(qp, qn, out=out, **dsc)

    seq_ms = timed(sequential)
    for m in maps:
        m[0].close()
    graph_ms = eager_ms = 0.0
    errors, bt = 0, None
    if mine:
        batch = PhotonMapBatch()
        out = batch.outputs(descs, qoff, dev)
        if args.leaf or args.wpb or args.rounds or args.layout >= 0:   # a fixed setting (profiling runs)
            wide = args.layout == 2 if args.layout >= 0 else True
            batch.set_tuning(leaf_size=args.leaf or 32, warps_per_block=args.wpb or 4,
                             rounds_per_chunk=args.rounds or 8, wide=wide)
            bt = {"leaf_size": args.leaf or 32, "warps_per_block": args.wpb or 4,
                  "rounds_per_chunk": args.rounds or 8, "wide_tree": wide, "chosen_by": "command line"}
        else:
            t = batch.autotune(d_pos, d_pw, poff, descs, d_qp, d_qn, qoff, out)
            bt = {"leaf_size": t.leaf_size, "warps_per_block": t.warps_per_block,
                  "rounds_per_chunk": t.rounds_per_chunk, "wide_tree": t.kbuf_layout == 2,
                  "chosen_by": "pm_batch_autotune (rank 0)"}

        def eager():
            batch.build(d_pos, d_pw, poff)
            batch.query(descs, d_qp, d_qn, qoff, out=out)

        eager_ms = timed(eager)
        batch.capture(d_pos, d_pw, poff, descs, d_qp, d_qn, qoff, out)
        graph_ms = timed(lambda: batch.launch())
        errors = batch.info().device_errors
        batch.close()
    else:   # a rank without maps still takes every collective step
        timed(lambda: None)
        timed(lambda: None)
    seq_ms, eager_ms, graph_ms, errors = rank_max([seq_ms, eager_ms, graph_ms, float(errors)], dev)
    close_ranks(world)
    if rank != 0:
        return None
    return {
        "metric": "batched photon maps: kNN radiance estimates/s (build + query of all maps per step)",
        "value": Q_all / (graph_ms / 1000.0), "unit": "queries/s", "higher_is_better": True, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "scaling": "strong", "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batch: {args.maps} maps, {N_all:,} photons, {Q_all:,} queries (log-uniform sizes, "
                               f"seed 777), k in {{16,32,64,128}}, R=0.05, cone filter",
                   "maps": args.maps, "photons": N_all, "queries": Q_all,
                   "l2": "flushed between steps (256 MiB write, untimed)",
                   "parallelism": "one GPU" if world == 1 else f"maps by LPT over {world} ranks, no exchange",
                   "rank0_maps": len(mine), "rank0_photons": N, "rank0_queries": Q},
        "batched_graph_ms": graph_ms, "batched_eager_ms": eager_ms, "sequential_per_map_ms": seq_ms,
        "sequential_queries_per_s": Q_all / (seq_ms / 1000.0), "batched_eager_queries_per_s": Q_all / (eager_ms / 1000.0),
        "speedup_graph_over_sequential": seq_ms / graph_ms, "device_errors": int(errors),
        "clocks": clock_runs[-1] if clock_runs else None,
        "batch_tuning": bt,
    }


def run_extras(args) -> dict:
    """The other workloads' headline figures, measured after the default
    line's own timed region in the same process (one GPU):
      final_gather  config-2 queries Hilbert-sorted against taken as given
      batch         the 64-map batch (one graph) against 64 sequential per-map calls
      diff          forward and forward + adjoint of the differentiation workload,
                    then the gradient-descent run on the powers
    Each keeps its own clocks record."""
    import copy
    out = {}
    fg_cfg = workload_config("final_gather")
    a = copy.copy(args)
    a.no_cpu_baseline = True
    a.unsorted = False
    srt = run_ours(a, fg_cfg, light=True)
    a.unsorted = True
    uns = run_ours(a, fg_cfg, light=True)
    out["final_gather"] = {
        "workload": fg_cfg["workload"], "metric": "queries/s (build + query per step)",
        "sorted_queries_per_s": srt["value"], "unsorted_queries_per_s": uns["value"],
        "speedup_sorted_over_unsorted": srt["value"] / uns["value"],
        "sorted": srt, "unsorted": uns}
    b = run_batch(copy.copy(args))
    out["batch"] = {k: b[k] for k in ("config", "value", "unit", "batched_graph_ms", "batched_eager_ms",
                                      "sequential_per_map_ms", "sequential_queries_per_s",
                                      "speedup_graph_over_sequential", "device_errors", "clocks", "batch_tuning")}
    d = run_diff(copy.copy(args), workload_config("diff"))
    out["diff"] = {k: d[k] for k in ("config", "forward_ms", "forward_no_lists_ms", "backward_ms",
                                     "fwd_bwd_over_fwd", "fwd_bwd_over_fwd_no_lists", "gradient_descent", "clocks")}
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="plain", choices=["small", "plain", "final_gather", "diff", "batch", "icut"])
    ap.add_argument("--maps", type=int, default=64, help="maps of the batch workload")
    ap.add_argument("--unsorted", action="store_true", help="keep the queries in the given order")
    ap.add_argument("--division", choices=["queries", "replicas"], default=None,
                    help="N > 1, plain / final-gather workloads: divide one map's queries over the ranks "
                         "(the default) or run an independent replica per rank")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: skip the final-gather, batch and diff sub-measurements")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel setting")
    ap.add_argument("--gd-steps", type=int, default=200, help="gradient-descent steps of the diff workload")
    ap.add_argument("--leaf", type=int, default=0)
    ap.add_argument("--wpb", type=int, default=0)
    ap.add_argument("--rounds", type=int, default=0)
    ap.add_argument("--qpw", type=int, default=0, help="queries per warp (group layout)")
    ap.add_argument("--layout", type=int, default=-1, help="k-buffer layout: 0 heap, 1 group, 2 wide tree")
    ap.add_argument("--chunks", type=int, default=1, help="query chunks of the end-to-end host-buffer call")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    cfg = workload_config("plain" if args.config == "icut" else args.config) if args.config != "batch" else None
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        print(json.dumps(run_reference(args, cfg)), flush=True)
        return 0
    if args.config == "batch":
        res = run_batch(args)
        if res is not None:
            print(json.dumps(res), flush=True)
        return 0
    if args.config == "diff":
        res = run_diff(args, cfg)
        if res is not None:
            print(json.dumps(res), flush=True)
        return 0
    if args.config == "icut":
        res = run_icut(args, cfg)
        if res is not None:
            print(json.dumps(res), flush=True)
        return 0
    res = run_ours(args, cfg)
    if res is not None and args.config == "plain" and res["n_gpus"] == 1 and not args.no_extras:
        res.update(run_extras(args))
    if res is not None:
        print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
