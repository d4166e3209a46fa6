"""Multi-GPU division of the photon-map path: one process per GPU over
torch.distributed (NCCL between GPUs, gloo on the CPU).

The path divides three ways, none of which needs data from another rank
during the forward:

* replicas -- every rank builds and queries its own map (independent
  photon maps, e.g. frames or scenes); no exchange at all.
* batched maps -- the maps of one batch (KDTreePoint instances of different
  sizes) go to ranks by LPT, longest processing time first, over a cost of
  photons + queries; each rank builds and queries its maps as one batch.
* one map, queries divided -- every rank builds the same map (the photons
  are a replicated input, 32 B each) and answers a contiguous range of the
  queries.  The forward needs no exchange.  The adjoint is linear in the
  queries' upstream gradients, so each rank's dL/dpower and dL/dposition are
  partial sums over its own queries, and one all-reduce sums them: the one
  real exchange step of the path (both gradients in float64, 64 B per
  photon).
"""
from __future__ import annotations

import numpy as np


def lpt_assign(costs, world: int) -> list[list[int]]:
    """Maps per rank: maps in decreasing cost (ties: lower index first), each
    to the rank with the least load so far (ties: lower rank).  Deterministic,
    so every rank computes the same assignment without communicating; within
    a rank the maps keep their batch order.  LPT's makespan is at most
    (4/3 - 1/(3 world)) of the optimum."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, dtype=np.float64)
    if c.ndim != 1 or (c < 0).any() or not np.isfinite(c).all():
        raise ValueError("costs must be a 1-D array of finite non-negative numbers")
    order = sorted(range(len(c)), key=lambda i: (-c[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        load[r] += float(c[i])
        out[r].append(i)
    return [sorted(m) for m in out]


def map_costs(n_photons, n_queries) -> np.ndarray:
    """The LPT cost of a map: photons + queries (build and query both scale
    about linearly in them)."""
    return np.asarray(n_photons, dtype=np.float64) + np.asarray(n_queries, dtype=np.float64)


def query_range(nq: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of the queries rank answers: contiguous, sizes differing
    by at most one, lower ranks taking the remainder."""
    if world < 1 or not 0 <= rank < world or nq < 0:
        raise ValueError("need 0 <= rank < world and nq >= 0")
    base, extra = divmod(nq, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def allreduce_gradients(*grads, group=None):
    """Sums per-photon partial gradients (n, 4) float32 over the ranks in
    place: each is widened to float64, summed by one all-reduce, and rounded
    back once, so the result differs from a single-rank adjoint only by each
    rank's own rounding of its partial sum (<= world * 2^-24 of the largest
    partial).  None entries are skipped; a world of one returns at once.
    Every rank must call this with the same tensors' shapes, in the same
    order."""
    import torch
    import torch.distributed as dist
    live = [g for g in grads if g is not None]
    if not live or not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return grads
    wide = torch.cat([g.reshape(-1).double() for g in live])
    dist.all_reduce(wide, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for g in live:
        m = g.numel()
        g.copy_(wide[off:off + m].view_as(g).to(g.dtype))
        off += m
    return grads


def allreduce_scalars(values, group=None) -> list[float]:
    """Sum over ranks of a few float64 scalars (losses, line-search terms)."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return vals
    dev = None
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [float(v) for v in t.tolist()]
