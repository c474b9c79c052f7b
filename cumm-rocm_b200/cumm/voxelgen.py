"""Seeded synthetic voxel clouds for the benchmark workloads (numpy only).

* ``uniform_voxels``: N unique voxels drawn uniformly without replacement from
  a cubic grid (the 20k-in-64^3 correctness workload).
* ``lidar_voxels``: LiDAR-like clouds in a (z, y, x) = (41, 1600, 1408) grid:
  points on 8 random planar patches plus 20 Gaussian clusters (sigma 2 voxels),
  voxelised and deduplicated to exactly N voxels.  Builder choices (stated
  because the workload description leaves them open): the clusters are filled
  first (a sigma-2 blob holds only a few hundred distinct voxels, so they give
  a small share); the rest comes from square planar patches of side
  0.75 * sqrt(remaining / 8) voxels with random (mostly ground-like) normals,
  sampled at 4 points per voxel of area so the surfaces are dense; further
  patches are added until N voxels exist.
* ``lognormal_sizes``: voxel counts for batches of clouds.
No dataset items are used; everything is generated from the seed.
"""
from typing import List, Sequence, Tuple

import numpy as np

KITTI_SHAPE = (41, 1600, 1408)  # (z, y, x)


def uniform_voxels(n: int, grid: int = 64, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lin = np.sort(rng.choice(grid ** 3, n, replace=False))
    z = lin // (grid * grid)
    y = (lin // grid) % grid
    x = lin % grid
    return np.stack([np.zeros_like(lin), z, y, x], 1).astype(np.int32)


def _dedupe_keep_order(coords: np.ndarray, shape: Sequence[int]) -> np.ndarray:
    lin = (coords[:, 0].astype(np.int64) * shape[1] + coords[:, 1]) * shape[2] + coords[:, 2]
    _, first = np.unique(lin, return_index=True)
    return coords[np.sort(first)]


def lidar_voxels(n: int, shape: Tuple[int, int, int] = KITTI_SHAPE, seed: int = 0,
                 n_planes: int = 8, n_clusters: int = 20, sigma: float = 2.0,
                 batch: int = 0) -> np.ndarray:
    """Returns int32 [n, 4] (batch, z, y, x) sorted by linear index.

    20 Gaussian clusters (sigma voxels, 2 * n / 20 points each, capped by what
    a sigma-2 blob can hold) come first; the remaining voxels are taken plane
    by plane from dense planar patches (4 points per voxel of patch area), so
    surfaces stay dense; if 8 patches fall short, more patches are added."""
    rng = np.random.default_rng(seed)
    D, H, W = shape
    centers = np.stack([rng.uniform(0, D, n_clusters), rng.uniform(0, H, n_clusters),
                        rng.uniform(0, W, n_clusters)], 1)
    per = max(1, min(4000, (2 * n) // (20 * n_clusters) * 20))
    cl = (centers[:, None, :] + rng.normal(scale=sigma, size=(n_clusters, per, 3))).reshape(-1, 3)
    parts = [cl]
    remaining = n
    vox = np.zeros((0, 3), np.int64)

    def clip_dedupe(p):
        v = np.floor(p).astype(np.int64)
        ok = (v[:, 0] >= 0) & (v[:, 0] < D) & (v[:, 1] >= 0) & (v[:, 1] < H) & \
             (v[:, 2] >= 0) & (v[:, 2] < W)
        return _dedupe_keep_order(v[ok], shape)

    vox = clip_dedupe(cl)[: n]
    remaining = n - vox.shape[0]
    side = max(8.0, np.sqrt(max(remaining, 1) / n_planes) * 0.75)
    planes_made = 0
    while vox.shape[0] < n:
        center = np.array([rng.uniform(0, D), rng.uniform(0, H), rng.uniform(0, W)])
        normal = rng.normal(size=3)
        normal[0] *= 3.0  # mostly ground-like / tilted surfaces
        normal /= np.linalg.norm(normal)
        u = np.cross(normal, [0.0, 0.0, 1.0])
        if np.linalg.norm(u) < 1e-3:
            u = np.cross(normal, [0.0, 1.0, 0.0])
        u /= np.linalg.norm(u)
        v = np.cross(normal, u)
        m = int(4 * side * side)
        a = rng.uniform(-side / 2, side / 2, m)
        b = rng.uniform(-side / 2, side / 2, m)
        p = center + a[:, None] * u + b[:, None] * v
        vox = _dedupe_keep_order(np.concatenate([vox, clip_dedupe(p)], 0), shape)
        planes_made += 1
    vox = vox[:n]
    lin = (vox[:, 0] * H + vox[:, 1]) * W + vox[:, 2]
    vox = vox[np.argsort(lin, kind="stable")]
    out = np.empty((n, 4), np.int32)
    out[:, 0] = batch
    out[:, 1:] = vox
    return out


def lognormal_sizes(count: int, median: float, sigma: float, lo: int, hi: int,
                    seed: int = 0) -> List[int]:
    rng = np.random.default_rng(seed)
    s = rng.lognormal(mean=np.log(median), sigma=sigma, size=count)
    return [int(x) for x in np.clip(np.round(s), lo, hi)]


def kaiming_uniform(K: int, kv: int, C: int, seed: int = 0) -> np.ndarray:
    """[K, kv, C] weights, U(-b, b) with b = sqrt(6 / (kv * C))."""
    rng = np.random.default_rng(seed)
    b = np.sqrt(6.0 / (kv * C))
    return rng.uniform(-b, b, size=(K, kv, C)).astype(np.float32)


def normal_features(n: int, C: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, C)).astype(np.float32)
