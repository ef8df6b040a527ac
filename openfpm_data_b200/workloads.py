"""Seeded synthetic workloads of the benchmark configurations.

Every generator uses numpy's PCG64 (``numpy.random.default_rng``) with the
configuration's seed; geometry and values draw from independent child
streams of ``SeedSequence(seed)`` unless stated otherwise.  Points are
returned as int64 [n, 3] (x, y, z) in z-major, x-fastest order.

  heat_shell   128^3, spherical shell 20 <= r <= 32 about (64,64,64),
               u ~ U[0,1) (seed 0), dt = 0.1, 100 steps
  gray_scott   512^3, union of 40 balls, centres U[0,512)^3, radii U[16,48]
               (seed 1); u = 1, v = 0, 6^3 cube at each centre u = 0.5,
               v = 0.25 with +-1 % uniform noise; Du .16 Dv .08 F .035
               k .065 dt 1, 1000 steps
  insert_batch 1024^3, 2M points per iteration: 70 % draws around 64
               Gaussian clusters (sigma 24), 30 % exact repeats (seed 2)
  batch_grids  256 grids, edge log-uniform in [32, 384] rounded to 8, one
               ball of radius U[0.25, 0.5] * edge (seed 3), heat rule
  requests     Poisson arrivals (seed 4), heat or Gray-Scott 50/50, edge
               log-uniform in [32, 256], 1-8 balls of radius U[0.1, 0.3] *
               edge, steps U[50, 500]
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HEAT_DT = 0.1
GS_PARAMS = dict(Du=0.16, Dv=0.08, F=0.035, k=0.065, dt=1.0)


def _streams(seed: int, n: int = 2):
    return [np.random.default_rng(s) for s in np.random.SeedSequence(seed).spawn(n)]


def ball_mask(size: Sequence[int], centres: np.ndarray, radii: np.ndarray) -> np.ndarray:
    """Boolean occupancy [z, y, x]: points with |p - c|^2 <= r^2 for some ball."""
    sz = [int(s) for s in size]
    occ = np.zeros((sz[2], sz[1], sz[0]), dtype=bool)
    for c, r in zip(centres, radii):
        lo = [max(0, int(np.floor(c[d] - r))) for d in range(3)]
        hi = [min(sz[d], int(np.ceil(c[d] + r)) + 1) for d in range(3)]
        if any(h <= l for l, h in zip(lo, hi)):
            continue
        z = np.arange(lo[2], hi[2])[:, None, None]
        y = np.arange(lo[1], hi[1])[None, :, None]
        x = np.arange(lo[0], hi[0])[None, None, :]
        d2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
        occ[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] |= d2 <= r * r
    return occ


def occupancy_points(occ: np.ndarray) -> np.ndarray:
    z, y, x = np.nonzero(occ)
    return np.stack([x, y, z], axis=1).astype(np.int64)


@dataclass
class PointSet:
    size: tuple
    coords: np.ndarray                 # int64 [n, 3]
    values: List[np.ndarray]           # one float32 array per field
    bck: List[float] = field(default_factory=lambda: [0.0])


def heat_shell(size: int = 128, r_in: float = 20.0, r_out: float = 32.0, seed: int = 0) -> PointSet:
    c = size // 2
    ax = np.arange(size)
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    d2 = (x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2
    occ = (d2 >= r_in * r_in) & (d2 <= r_out * r_out)
    pts = occupancy_points(occ)
    rng = np.random.default_rng(seed)
    u = rng.random(len(pts), dtype=np.float32)
    return PointSet((size, size, size), pts, [u], [0.0])


def gray_scott(size: int = 512, nballs: int = 40, rmin: float = 16.0, rmax: float = 48.0, seed: int = 1,
               cube: int = 6, noise: float = 0.01) -> PointSet:
    geo, val = _streams(seed)
    centres = geo.uniform(0, size, size=(nballs, 3))
    radii = geo.uniform(rmin, rmax, size=nballs)
    occ = ball_mask((size, size, size), centres, radii)
    # the seeded cubes are set on a dense index so overlaps resolve in ball order
    uz = np.ones(occ.shape, dtype=np.float32)
    vz = np.zeros(occ.shape, dtype=np.float32)
    h = cube // 2
    for c in centres:
        ci = np.floor(c).astype(int)
        lo = np.maximum(ci - h, 0)
        hi = np.minimum(ci + (cube - h), size)
        shp = (hi[2] - lo[2], hi[1] - lo[1], hi[0] - lo[0])
        nu = val.uniform(-1.0, 1.0, size=shp).astype(np.float32)
        nv = val.uniform(-1.0, 1.0, size=shp).astype(np.float32)
        uz[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = np.float32(0.5) * (np.float32(1.0) + np.float32(noise) * nu)
        vz[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = np.float32(0.25) * (np.float32(1.0) + np.float32(noise) * nv)
    pts = occupancy_points(occ)
    u = uz[pts[:, 2], pts[:, 1], pts[:, 0]]
    v = vz[pts[:, 2], pts[:, 1], pts[:, 0]]
    return PointSet((size, size, size), pts, [u, v], [1.0, 0.0])


def insert_batch(iteration: int, npts: int = 2_000_000, size: int = 1024, nclusters: int = 64, sigma: float = 24.0,
                 dup_frac: float = 0.3, seed: int = 2):
    """One iteration of the insert/flush stress test: coords int64 [n,3],
    float32 payload, int32 payload.  Cluster centres are fixed by the seed,
    draws differ per iteration."""
    cen_rng = np.random.default_rng(np.random.SeedSequence(seed).spawn(1)[0])
    centres = cen_rng.uniform(0, size, size=(nclusters, 3))
    rng = np.random.default_rng(np.random.SeedSequence([seed, iteration + 1]))
    nfresh = npts - int(round(npts * dup_frac))
    which = rng.integers(0, nclusters, size=nfresh)
    pts = np.rint(centres[which] + rng.normal(0.0, sigma, size=(nfresh, 3)))
    pts = np.clip(pts, 0, size - 1).astype(np.int64)
    ndup = npts - nfresh
    src = rng.integers(0, nfresh, size=ndup)
    allp = np.concatenate([pts, pts[src]], axis=0)
    order = rng.permutation(npts)   # duplicates interleave with the originals
    allp = allp[order]
    fval = rng.random(npts, dtype=np.float32)
    ival = rng.integers(-(2 ** 31), 2 ** 31 - 1, size=npts, dtype=np.int64).astype(np.int32)
    return allp, fval, ival


def batch_grids(ngrids: int = 256, emin: int = 32, emax: int = 384, seed: int = 3, rfrac=(0.25, 0.5)):
    """Edges and ball radii of the batched configuration."""
    rng = np.random.default_rng(seed)
    edges = np.exp(rng.uniform(np.log(emin), np.log(emax), size=ngrids))
    edges = np.clip((np.rint(edges / 8) * 8).astype(int), emin, emax)
    radii = rng.uniform(rfrac[0], rfrac[1], size=ngrids) * edges
    vals_seed = rng.integers(0, 2 ** 31, size=ngrids)
    return edges, radii, vals_seed


def single_ball_grid(edge: int, radius: float, vseed: int) -> PointSet:
    c = np.array([[edge / 2.0] * 3])
    occ = ball_mask((edge, edge, edge), c, np.array([radius]))
    pts = occupancy_points(occ)
    u = np.random.default_rng(int(vseed)).random(len(pts), dtype=np.float32)
    return PointSet((edge, edge, edge), pts, [u], [0.0])


@dataclass
class Request:
    rid: int
    t_arrival: float
    kind: str          # "heat" or "gs"
    edge: int
    centres: np.ndarray
    radii: np.ndarray
    steps: int
    vseed: int


def requests(rate: float = 2000.0, duration: float = 60.0, seed: int = 4, emin: int = 32, emax: int = 256,
             rfrac=(0.1, 0.3), steps=(50, 500), limit: Optional[int] = None) -> List[Request]:
    rng = np.random.default_rng(seed)
    out: List[Request] = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (limit is not None and len(out) >= limit):
            break
        kind = "heat" if rng.random() < 0.5 else "gs"
        edge = int(np.clip(np.rint(np.exp(rng.uniform(np.log(emin), np.log(emax))) / 8) * 8, emin, emax))
        nb = int(rng.integers(1, 9))
        cen = rng.uniform(0, edge, size=(nb, 3))
        rad = rng.uniform(rfrac[0], rfrac[1], size=nb) * edge
        st = int(rng.integers(steps[0], steps[1] + 1))
        out.append(Request(len(out), t, kind, edge, cen, rad, st, int(rng.integers(0, 2 ** 31))))
    return out


def request_points(req: Request) -> PointSet:
    occ = ball_mask((req.edge,) * 3, req.centres, req.radii)
    pts = occupancy_points(occ)
    rng = np.random.default_rng(req.vseed)
    if req.kind == "heat":
        return PointSet((req.edge,) * 3, pts, [rng.random(len(pts), dtype=np.float32)], [0.0])
    u = np.ones(len(pts), np.float32)
    v = np.zeros(len(pts), np.float32)
    # seed v (and dent u) in a 6^3 cube around each ball centre
    for c in req.centres:
        ci = np.floor(c).astype(np.int64)
        inside = np.all((pts - ci >= -3) & (pts - ci <= 2), axis=1)
        u[inside] = np.float32(0.5) * (np.float32(1) + np.float32(0.01) * rng.uniform(-1, 1, inside.sum()).astype(np.float32))
        v[inside] = np.float32(0.25) * (np.float32(1) + np.float32(0.01) * rng.uniform(-1, 1, inside.sum()).astype(np.float32))
    return PointSet((req.edge,) * 3, pts, [u, v], [1.0, 0.0])


def build_block_map(coords: np.ndarray, values: Sequence[np.ndarray], size: Sequence[int], edge: int,
                    bck: Optional[Sequence[float]] = None):
    """Host construction of a block map (grid_smb layout) from unique points:
    returns keys[n] (sorted), data arrays [n*bs] per field, mask[n*bs].
    Points absent from a chunk hold the background value and mask 0."""
    coords = np.asarray(coords, dtype=np.int64)
    bsz = [(int(s) + edge - 1) // edge for s in size]
    b = ((coords[:, 2] // edge) * bsz[1] + coords[:, 1] // edge) * bsz[0] + coords[:, 0] // edge
    l = ((coords[:, 2] % edge) * edge + coords[:, 1] % edge) * edge + coords[:, 0] % edge
    keys, inv = np.unique(b, return_inverse=True)
    bs = edge ** 3
    idx = inv * bs + l
    n = len(keys)
    bck = bck or [0.0] * len(values)
    data = []
    for v, bv in zip(values, bck):
        d = np.full(n * bs, bv, dtype=np.asarray(v).dtype)
        d[idx] = v
        data.append(d)
    mask = np.zeros(n * bs, dtype=np.uint8)
    mask[idx] = 1
    return keys.astype(np.int64), data, mask
