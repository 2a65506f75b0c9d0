"""Seeded synthetic NDT workloads (plane + vertical walls), one per benchmark config.

The DAPHNE ndt_mapping input set (data/ndt_input.dat) is not available, so the
workloads are generated: a ground plane z = 0 with ~N(0, 0.02 m) noise plus K
vertical walls (centre uniform in the area, random heading, length U(2, 10) m,
height U(1, 4) m, the same noise across the wall), sampled uniformly by surface
area.  A scan is a fresh sample of the same surfaces within 40 m of a sensor
pose (xy uniform in the inner half of the area, any yaw, z = 0), expressed in
the sensor frame; the guess is the ground truth perturbed by uniform +-dt in x,
y and +-dyaw in yaw.  Points are float32 (x, y, z, 1); a scan's points are
ordered like a voxel-grid filtered scan (by 2 m leaf index, x fastest).

Reproducibility: only IEEE basic arithmetic (+ - * / and comparisons) is applied
to random numbers -- headings come from the rational parametrisation
(cos, sin) = ((1 - t^2) / (1 + t^2), 2t / (1 + t^2)), noise is a scaled sum of
four uniforms (Irwin-Hall), the yaw perturbation is 2 atan(t) with t uniform in
+-tan(dyaw / 2) -- so a seed yields the same bytes on every machine.
"""
from __future__ import annotations

import dataclasses
import hashlib
import math

import numpy as np

SQRT3 = 1.7320508075688772
# tan(d / 2) for the yaw perturbation bounds used below (d in degrees).
_TAN_HALF_DEG = {
    3.0: 0.02618592156918693,
    5.0: 0.04366094290851206,
    10.0: 0.08748866352592401,
    15.0: 0.13165249758739583,
}


@dataclasses.dataclass(frozen=True)
class Config:
    """One benchmark configuration (sizes and perturbations)."""

    name: str
    map_points: int
    area: float
    walls: int
    resolution: float
    aligns: int
    scan_min: int
    scan_max: int
    log_uniform: bool
    dt: float
    dyaw_deg: float
    radius: float = 40.0
    seed: int = 0


CONFIGS = {
    # one alignment, CPU-runnable: 60k map over 60 x 60 m, 30 walls, 2k scan
    "c1": Config("c1", 60_000, 60.0, 30, 1.0, 1, 2000, 2000, False, 0.5, 3.0, seed=1000),
    # benchmark scale: 400k map over 150 x 150 m, 120 walls, 256 x 8k scans
    "c2": Config("c2", 400_000, 150.0, 120, 1.0, 256, 8000, 8000, False, 0.5, 3.0, seed=2000),
    # batched: c2 map, 1024 scans log-uniform in 1k-16k, +-1 m / +-5 deg
    "c3": Config("c3", 400_000, 150.0, 120, 1.0, 1024, 1000, 16000, True, 1.0, 5.0, seed=2000),
    # learned-init training pairs: c2 map, +-2 m / +-10 deg
    "c4": Config("c4", 400_000, 150.0, 120, 1.0, 1024, 2000, 8000, True, 2.0, 10.0, seed=2000),
    # large: 2M map over 300 x 300 m, 400 walls, res 0.5, 4096 scans in 2k-32k
    "c5": Config("c5", 2_000_000, 300.0, 400, 0.5, 4096, 2000, 32000, True, 3.0, 15.0, seed=5000),
}


@dataclasses.dataclass
class Scene:
    """Map surfaces and the sampled map cloud."""

    area: float
    walls: np.ndarray  # (K, 7): cx, cy, dx, dy, length, height, area
    map: np.ndarray  # (M, 4) float32


@dataclasses.dataclass
class Alignment:
    scan: np.ndarray  # (N, 4) float32, sensor frame
    guess: np.ndarray  # (16,) float32, row-major 4x4
    truth: np.ndarray  # (4, 4) float64 ground-truth sensor pose


def _unit(t):
    d = 1.0 + t * t
    return (1.0 - t * t) / d, (2.0 * t) / d


def _noise(rng, n, sigma):
    u = rng.random((n, 4))
    return ((u[:, 0] + u[:, 1] + u[:, 2] + u[:, 3]) - 2.0) * (SQRT3 * sigma)


def _wall_points(rng, walls, idx, sigma):
    n = idx.shape[0]
    w = walls[idx]
    s = (rng.random(n) - 0.5) * w[:, 4]
    h = rng.random(n) * w[:, 5]
    e = _noise(rng, n, sigma)
    x = w[:, 0] + s * w[:, 2] - e * w[:, 3]
    y = w[:, 1] + s * w[:, 3] + e * w[:, 2]
    return np.stack([x, y, h], axis=1)


def make_scene(cfg: Config, sigma: float = 0.02) -> Scene:
    """Map cloud of `cfg.map_points` points (seed cfg.seed)."""
    rng = np.random.default_rng([cfg.seed, 0])
    W = cfg.area
    K = cfg.walls
    c = (rng.random((K, 2)) - 0.5) * W
    dx, dy = _unit(rng.random(K) * 2.0 - 1.0)
    length = 2.0 + rng.random(K) * 8.0
    height = 1.0 + rng.random(K) * 3.0
    walls = np.stack([c[:, 0], c[:, 1], dx, dy, length, height, length * height], axis=1)
    a_ground = W * W
    a_walls = math.fsum(walls[:, 6].tolist())
    n_ground = int(np.floor(cfg.map_points * (a_ground / (a_ground + a_walls)) + 0.5))
    n_walls = cfg.map_points - n_ground
    g = (rng.random((n_ground, 2)) - 0.5) * W
    gz = _noise(rng, n_ground, sigma)
    ground = np.stack([g[:, 0], g[:, 1], gz], axis=1)
    cum = np.cumsum(walls[:, 6])
    pick = np.searchsorted(cum, rng.random(n_walls) * cum[-1], side="right")
    pick = np.minimum(pick, K - 1)
    wp = _wall_points(rng, walls, pick, sigma)
    pts = np.concatenate([ground, wp], axis=0)
    perm = rng.permutation(pts.shape[0])
    pts = pts[perm]
    out = np.ones((pts.shape[0], 4), dtype=np.float32)
    out[:, :3] = pts.astype(np.float32)
    return Scene(area=W, walls=walls, map=out)


def _scan_world(rng, scene: Scene, sx, sy, n, radius, sigma):
    """n surface samples within `radius` of (sx, sy, 0), area-weighted."""
    W = scene.area
    half = W / 2.0
    x0, x1 = max(-half, sx - radius), min(half, sx + radius)
    y0, y1 = max(-half, sy - radius), min(half, sy + radius)
    a_ground = (x1 - x0) * (y1 - y0)
    walls = scene.walls
    reach = radius + 6.0
    near = np.nonzero((walls[:, 0] - sx) ** 2 + (walls[:, 1] - sy) ** 2 < reach * reach)[0]
    wsub = walls[near]
    a_walls = math.fsum(wsub[:, 6].tolist()) if near.size else 0.0
    p_ground = a_ground / (a_ground + a_walls)
    got = []
    have = 0
    while have < n:
        m = max(256, int((n - have) * 1.6))
        is_g = rng.random(m) < p_ground
        ng = int(np.count_nonzero(is_g))
        nw = m - ng
        u = rng.random((ng, 2))
        gx = x0 + u[:, 0] * (x1 - x0)
        gy = y0 + u[:, 1] * (y1 - y0)
        gz = _noise(rng, ng, sigma)
        parts = [np.stack([gx, gy, gz], axis=1)]
        if nw and near.size:
            cum = np.cumsum(wsub[:, 6])
            pick = np.minimum(np.searchsorted(cum, rng.random(nw) * cum[-1], side="right"), near.size - 1)
            parts.append(_wall_points(rng, wsub, pick, sigma))
        cand = np.concatenate(parts, axis=0)
        order = rng.permutation(cand.shape[0])
        cand = cand[order]
        d2 = (cand[:, 0] - sx) ** 2 + (cand[:, 1] - sy) ** 2 + cand[:, 2] ** 2
        keep = cand[d2 < radius * radius]
        got.append(keep)
        have += keep.shape[0]
    return np.concatenate(got, axis=0)[:n]


def make_alignment(cfg: Config, scene: Scene, index: int, n_points: int | None = None,
                   sigma: float = 0.02) -> Alignment:
    """Scan, guess and ground truth of alignment `index` (seeded by cfg.seed, index)."""
    rng = np.random.default_rng([cfg.seed, 1, index])
    W = cfg.area
    if n_points is None:
        n_points = scan_size(cfg, index)
    sx, sy = (rng.random(2) - 0.5) * (W / 2.0)
    c, s = _unit(rng.random() * 2.0 - 1.0)
    if rng.random() < 0.5:
        c, s = -c, -s
    world = _scan_world(rng, scene, sx, sy, n_points, cfg.radius, sigma)
    # sensor frame: R^T (p - t)
    px, py, pz = world[:, 0] - sx, world[:, 1] - sy, world[:, 2]
    lx = c * px + s * py
    ly = -s * px + c * py
    scan = np.ones((n_points, 4), dtype=np.float32)
    scan[:, 0] = lx.astype(np.float32)
    scan[:, 1] = ly.astype(np.float32)
    scan[:, 2] = pz.astype(np.float32)
    scan = scan[leaf_order(scan)]
    truth = np.eye(4)
    truth[0, 0], truth[0, 1], truth[1, 0], truth[1, 1] = c, -s, s, c
    truth[0, 3], truth[1, 3] = sx, sy
    th = _TAN_HALF_DEG[cfg.dyaw_deg]
    dc, ds = _unit((rng.random() * 2.0 - 1.0) * th)
    gc, gs = c * dc - s * ds, s * dc + c * ds
    ex, ey = (rng.random(2) * 2.0 - 1.0) * cfg.dt
    guess = np.eye(4)
    guess[0, 0], guess[0, 1], guess[1, 0], guess[1, 1] = gc, -gs, gs, gc
    guess[0, 3], guess[1, 3] = sx + ex, sy + ey
    return Alignment(scan=scan, guess=guess.astype(np.float32).reshape(16), truth=truth)


def make_raw_scan(cfg: Config, scene: Scene, index: int, n_points: int, radius: float = 60.0,
                  sigma: float = 0.02) -> np.ndarray:
    """An unfiltered scan of alignment `index`'s sensor pose: n_points surface
    samples within `radius` in the sensor frame, in sweep order (by azimuth),
    intensity uniform in [0, 255) -- the input of the voxel-grid pre-filter."""
    rng = np.random.default_rng([cfg.seed, 3, index])
    W = cfg.area
    sx, sy = (rng.random(2) - 0.5) * (W / 2.0)
    world = _scan_world(rng, scene, sx, sy, n_points, radius, sigma)
    px, py = world[:, 0] - sx, world[:, 1] - sy
    scan = np.empty((n_points, 4), dtype=np.float32)
    scan[:, 0] = px.astype(np.float32)
    scan[:, 1] = py.astype(np.float32)
    scan[:, 2] = world[:, 2].astype(np.float32)
    scan[:, 3] = (rng.random(n_points) * 255.0).astype(np.float32)
    return scan[np.argsort(np.arctan2(py, px), kind="stable")]


def leaf_order(scan, leaf=2.0):
    """Point order of a voxel-grid filtered scan: by 2 m leaf index, x fastest.

    The align call's input is a "filtered_scan" (a voxel-grid downsampled
    LiDAR scan), whose points come out ordered by leaf index; this reproduces
    that order (stable integer sort, machine independent).
    """
    q = np.floor(scan[:, :3].astype(np.float64) / leaf).astype(np.int64) + 1024
    key = (q[:, 2] * 2048 + q[:, 1]) * 2048 + q[:, 0]
    return np.argsort(key, kind="stable")


def scan_size(cfg: Config, index: int) -> int:
    """Scan size of alignment `index`: fixed, or log-uniform in [scan_min, scan_max]."""
    if not cfg.log_uniform:
        return cfg.scan_min
    rng = np.random.default_rng([cfg.seed, 2, index])
    lo, hi = np.log(cfg.scan_min), np.log(cfg.scan_max)
    return int(np.clip(np.floor(np.exp(lo + rng.random() * (hi - lo)) + 0.5), cfg.scan_min, cfg.scan_max))


def make_batch(cfg: Config, count: int | None = None, start: int = 0, scene: Scene | None = None):
    """Scene plus `count` alignments (default cfg.aligns) starting at `start`."""
    if scene is None:
        scene = make_scene(cfg)
    count = cfg.aligns if count is None else count
    return scene, [make_alignment(cfg, scene, start + i) for i in range(count)]


def small_config(name: str, map_points: int, area: float, walls: int, scan: int, seed: int,
                 resolution: float = 1.0, dt: float = 0.5, dyaw_deg: float = 3.0,
                 radius: float = 40.0) -> Config:
    """A reduced configuration with the same generator (tests)."""
    return Config(name, map_points, area, walls, resolution, 1, scan, scan, False, dt, dyaw_deg,
                  radius=radius, seed=seed)


def digest(*arrays) -> str:
    """sha256 over the raw bytes of arrays (fixture reproducibility check)."""
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()
