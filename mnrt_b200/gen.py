"""Seeded synthetic photon maps and query sets (numpy, host side).

The workloads stand in for MNRT's photon tracing (GPU/photon_build.cu) and
gather-ray hits (GPU/raygen.cu, GPU/raytracing.cu), which are outside the
engine.  Shapes follow the benchmark configurations:

  room       the unit-cube room: floor y=0, ceiling y=1, walls x=0, x=1 and
             z=0 (z=1 is open); a uniform wall point = a uniform wall (equal
             areas) then a uniform (u, v) on it
  caustic    a fraction of the photons from N((0.5, 0, 0.5), sigma) on the
             floor, (x, z) clamped to [0, 1]
  power      each RGB channel Exponential(mean = power_mean)
  direction  travel direction d = -(cosine-weighted sample about the wall's
             inward normal), so the photon's own wall sees dot(n, -d) > 0
  queries    uniform wall points with the inward normal; optionally a mix with
             Gaussian clusters (sigma) on the walls, shuffled

Every array is float32.  Photons come in two layouts: "packed" (the engine's
native record: pos.w unused, pow.w = octahedral direction bits) and
"reference" (MNRT's PhotonData: pos.w = azimuth phi, pow.w = polar theta).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# (axis held constant, its value, inward normal)
WALLS = (
    (1, 0.0, (0.0, 1.0, 0.0)),   # floor
    (1, 1.0, (0.0, -1.0, 0.0)),  # ceiling
    (0, 0.0, (1.0, 0.0, 0.0)),   # x = 0
    (0, 1.0, (-1.0, 0.0, 0.0)),  # x = 1
    (2, 0.0, (0.0, 0.0, 1.0)),   # z = 0
)


@dataclass
class PhotonSet:
    pos: np.ndarray      # (n, 4) float32; w per layout
    pow: np.ndarray      # (n, 4) float32; w per layout
    dirs: np.ndarray     # (n, 3) float32 travel directions
    layout: str          # "packed" or "reference"

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


@dataclass
class QuerySet:
    pos: np.ndarray      # (nq, 4) float32, w = 0
    nrm: np.ndarray      # (nq, 4) float32, w = 0

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def _wall_points(rng: np.random.Generator, n: int):
    w = rng.integers(0, len(WALLS), size=n)
    uv = rng.random((n, 2))
    p = np.empty((n, 3), np.float64)
    nrm = np.empty((n, 3), np.float64)
    for i, (axis, val, nv) in enumerate(WALLS):
        m = w == i
        others = [a for a in range(3) if a != axis]
        p[m, axis] = val
        p[m, others[0]] = uv[m, 0]
        p[m, others[1]] = uv[m, 1]
        nrm[m] = nv
    return p, nrm, w


def _cosine_about(rng: np.random.Generator, nrm: np.ndarray) -> np.ndarray:
    n = nrm.shape[0]
    u1, u2 = rng.random(n), rng.random(n)
    r, phi = np.sqrt(u1), 2.0 * np.pi * u2
    lx, ly, lz = r * np.cos(phi), r * np.sin(phi), np.sqrt(np.maximum(0.0, 1.0 - u1))
    # tangent frame: pick a helper axis not parallel to the normal
    helper = np.where(np.abs(nrm[:, :1]) > 0.5, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    t = np.cross(helper, nrm)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(nrm, t)
    return lx[:, None] * t + ly[:, None] * b + lz[:, None] * nrm


def oct_encode(d: np.ndarray) -> np.ndarray:
    """Octahedral code of float32 directions, same FP32 steps as the engine."""
    d = d.astype(np.float32)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    s = (np.abs(x) + np.abs(y)) + np.abs(z)
    with np.errstate(divide="ignore", invalid="ignore"):
        px, py = x / s, y / s
    one = np.float32(1.0)
    sx = np.where(px >= 0, one, -one).astype(np.float32)
    sy = np.where(py >= 0, one, -one).astype(np.float32)
    fx = ((one - np.abs(py)) * sx).astype(np.float32)
    fy = ((one - np.abs(px)) * sy).astype(np.float32)
    neg = z < 0
    px = np.where(neg, fx, px).astype(np.float32)
    py = np.where(neg, fy, py).astype(np.float32)
    px = np.where(s > 0, px, np.float32(0)).astype(np.float32)
    py = np.where(s > 0, py, np.float32(0)).astype(np.float32)
    k = np.float32(32767.0)
    u = np.clip(np.rint((px * k).astype(np.float32)), -32767, 32767).astype(np.int32)
    v = np.clip(np.rint((py * k).astype(np.float32)), -32767, 32767).astype(np.int32)
    bits = (u.astype(np.uint32) & 0xFFFF) | ((v.astype(np.uint32) & 0xFFFF) << 16)
    bits = np.where(s > 0, bits, 0).astype(np.uint32)
    return bits


def oct_decode(bits: np.ndarray) -> np.ndarray:
    """Unnormalised direction from octahedral codes (engine's FP32 steps)."""
    bits = np.asarray(bits, np.uint32)
    iu = (bits & 0xFFFF).astype(np.uint16).view(np.int16).astype(np.float32)
    iv = (bits >> 16).astype(np.uint16).view(np.int16).astype(np.float32)
    s = np.float32(1.0) / np.float32(32767.0)
    fu, fv = (iu * s).astype(np.float32), (iv * s).astype(np.float32)
    au, av = np.abs(fu), np.abs(fv)
    one = np.float32(1.0)
    z = ((one - au) - av).astype(np.float32)
    x = np.where(z < 0, (one - av) * np.where(fu >= 0, one, -one), fu).astype(np.float32)
    y = np.where(z < 0, (one - au) * np.where(fv >= 0, one, -one), fv).astype(np.float32)
    return np.stack([x, y, z], axis=1).astype(np.float32)


def photons(n: int, seed: int, caustic_frac: float = 0.2, caustic_sigma: float = 0.01,
            power_mean: float | None = None, layout: str = "packed") -> PhotonSet:
    rng = np.random.default_rng(seed)
    nc = int(round(n * caustic_frac))
    nu = n - nc
    p, nrm, _ = _wall_points(rng, nu)
    if nc:
        c = rng.normal(0.0, caustic_sigma, size=(nc, 2))
        cp = np.zeros((nc, 3))
        cp[:, 0] = np.clip(0.5 + c[:, 0], 0.0, 1.0)
        cp[:, 2] = np.clip(0.5 + c[:, 1], 0.0, 1.0)
        cn = np.tile(np.array([[0.0, 1.0, 0.0]]), (nc, 1))
        p = np.concatenate([p, cp])
        nrm = np.concatenate([nrm, cn])
        perm = rng.permutation(n)      # caustic photons interleaved with the rest
        p, nrm = p[perm], nrm[perm]
    travel = -_cosine_about(rng, nrm)
    mean = power_mean if power_mean is not None else 1.0 / max(n, 1)
    flux = rng.exponential(mean, size=(n, 3))
    pos = np.zeros((n, 4), np.float32)
    pw = np.zeros((n, 4), np.float32)
    pos[:, :3] = p
    pw[:, :3] = flux
    dirs = travel.astype(np.float32)
    if layout == "packed":
        pw[:, 3] = oct_encode(dirs).view(np.float32)
    elif layout == "reference":
        d64 = dirs.astype(np.float64)
        d64 /= np.linalg.norm(d64, axis=1, keepdims=True)
        phi = np.arctan2(d64[:, 1], d64[:, 0])
        phi = np.where(phi < 0, phi + 2 * np.pi, phi)
        theta = np.arccos(np.clip(d64[:, 2], -1.0, 1.0))
        pos[:, 3] = phi.astype(np.float32)
        pw[:, 3] = theta.astype(np.float32)
    else:
        raise ValueError(layout)
    return PhotonSet(pos, pw, dirs, layout)


def queries(nq: int, seed: int, cluster_frac: float = 0.0, clusters: int = 64,
            cluster_sigma: float = 0.02) -> QuerySet:
    rng = np.random.default_rng(seed)
    ncl = int(round(nq * cluster_frac))
    nu = nq - ncl
    p, nrm, _ = _wall_points(rng, nu)
    if ncl:
        cp, cn, cw = _wall_points(rng, clusters)
        which = rng.integers(0, clusters, size=ncl)
        q = cp[which].copy()
        off = rng.normal(0.0, cluster_sigma, size=(ncl, 2))
        for i, (axis, _val, _nv) in enumerate(WALLS):
            m = cw[which] == i
            others = [a for a in range(3) if a != axis]
            q[m, others[0]] = np.clip(q[m, others[0]] + off[m, 0], 0.0, 1.0)
            q[m, others[1]] = np.clip(q[m, others[1]] + off[m, 1], 0.0, 1.0)
        p = np.concatenate([p, q])
        nrm = np.concatenate([nrm, cn[which]])
        perm = rng.permutation(nq)
        p, nrm = p[perm], nrm[perm]
    pos = np.zeros((nq, 4), np.float32)
    nn = np.zeros((nq, 4), np.float32)
    pos[:, :3] = p
    nn[:, :3] = nrm
    return QuerySet(pos, nn)


@dataclass
class BatchSpec:
    n: list
    nq: list
    k: list
    seeds: list


def batch_spec(num_maps: int, seed: int, n_range=(1e4, 2e6), q_range=(1e3, 1e6), ks=(16, 32, 64, 128)) -> BatchSpec:
    """Per-map sizes: photon and query counts log-uniform, k uniform over ks."""
    rng = np.random.default_rng(seed)
    n = np.floor(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]), num_maps))).astype(int)
    q = np.floor(np.exp(rng.uniform(np.log(q_range[0]), np.log(q_range[1]), num_maps))).astype(int)
    k = rng.choice(np.array(ks), size=num_maps)
    return BatchSpec([int(x) for x in n], [int(x) for x in q], [int(x) for x in k],
                     [seed + 1000 + i for i in range(num_maps)])


# Named workloads (photons, queries, k, R, filter).
CONFIGS = {
    "small": dict(n=65536, nq=16384, k=50, r_max=0.1, filter="cone", caustic_frac=0.0, power_mean=1.0 / 65536),
    "plain": dict(n=1048576, nq=2073600, k=100, r_max=0.05, filter="cone", caustic_frac=0.2),
    "final_gather": dict(n=4194304, nq=8388608, k=64, r_max=0.05, filter="cone", caustic_frac=0.2, cluster_frac=0.5),
    "diff": dict(n=1048576, nq=1048576, k=64, r_max=0.05, filter="epanechnikov", caustic_frac=0.2),
}
