"""Seeded synthetic point clouds for the benchmark configurations.

They stand in for the S3DIS / SemanticKITTI crops the reference measures on
(those datasets are not redistributed).  Every generator is deterministic in
its seed (47 by default, the reference's seed: FlashKNN/test.py:29).  The
cube and room clouds are voxel-first deduplicated at the grid voxel like the
reference's benchmark preparation (Query/benchmark_s3dis.py:156-167); LiDAR
scans keep several returns per voxel in the near field.

  uniform_cube   C1  16,384 points in [0,1)^3, voxel 0.0197 (parent = 2x spacing)
  room           C2  ~80k points on a 6x8x3 m room + 10 boxes, sigma 5 mm, 4 cm voxels
  lidar          C3  64 rings x 2048 azimuths, ground + cylinders + boxes to 50 m,
                     10% dropped, 5 cm voxels
  uneven_batch   C4  16 clouds, counts log-uniform in [20k, 200k], room / lidar mixed,
                     every cloud voxel-first deduplicated at the 5 cm grid voxel
  backward_weights C5 w ~ N(0,1) for the loss sum(w * d)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SEED = 47


def voxel_first(xyz: np.ndarray, voxel: float) -> np.ndarray:
    """Keep the first point of every occupied voxel, in input order."""
    grid = np.floor(xyz / np.float32(voxel)).astype(np.int64)
    _, first = np.unique(grid, axis=0, return_index=True)
    return xyz[np.sort(first)]


def uniform_cube(n: int = 16384, seed: int = SEED, voxel: float = 0.0197) -> np.ndarray:
    rng = np.random.default_rng(seed)
    pts = np.zeros((0, 3), np.float32)
    while len(pts) < n:
        extra = rng.random((n, 3), dtype=np.float32)
        pts = voxel_first(np.concatenate([pts, extra]), voxel)
    return np.ascontiguousarray(pts[:n])


def _box_faces(lo, hi, n, rng):
    """n points on the 5 visible faces (no bottom) of an axis-aligned box."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    size = hi - lo
    areas = np.array([size[0] * size[1],              # top
                      size[1] * size[2], size[1] * size[2],
                      size[0] * size[2], size[0] * size[2]], np.float64)
    face = rng.choice(5, size=n, p=areas / areas.sum())
    u = rng.random(n, dtype=np.float32)
    v = rng.random(n, dtype=np.float32)
    pts = np.empty((n, 3), np.float32)
    top = face == 0
    pts[top] = np.stack([lo[0] + u[top] * size[0], lo[1] + v[top] * size[1],
                         np.full(top.sum(), hi[2], np.float32)], 1)
    for f, (axis, val) in enumerate([(0, lo[0]), (0, hi[0]), (1, lo[1]), (1, hi[1])], start=1):
        m = face == f
        o1, o2 = [a for a in range(3) if a != axis]
        pts[m, axis] = val
        pts[m, o1] = lo[o1] + u[m] * size[o1]
        pts[m, o2] = lo[o2] + v[m] * size[o2]
    return pts


def room(seed: int = SEED, target: int = 80000, voxel: float = 0.04, dims=(6.0, 8.0, 3.0),
         n_boxes: int = 10, noise: float = 0.005) -> np.ndarray:
    """Floor, ceiling, four walls and furniture boxes, 5 mm noise, voxel-first."""
    rng = np.random.default_rng(seed)
    W, L, H = dims
    planes = [  # (fixed axis, value, extent axes)
        (2, 0.0), (2, H), (0, 0.0), (0, W), (1, 0.0), (1, L)]
    ext = {0: W, 1: L, 2: H}
    areas = []
    for axis, _ in planes:
        o1, o2 = [a for a in range(3) if a != axis]
        areas.append(ext[o1] * ext[o2])
    boxes = []
    for _ in range(n_boxes):
        sx, sy = rng.uniform(0.4, 2.0, 2)
        sz = rng.uniform(0.4, 1.8)
        x0 = rng.uniform(0.1, W - sx - 0.1)
        y0 = rng.uniform(0.1, L - sy - 0.1)
        boxes.append(((x0, y0, 0.0), (x0 + sx, y0 + sy, sz)))
    box_area = sum((hi[0] - lo[0]) * (hi[1] - lo[1]) + 2 * (hi[2] - lo[2]) *
                   ((hi[0] - lo[0]) + (hi[1] - lo[1])) for lo, hi in boxes)
    total_area = sum(areas) + box_area
    # Raw sample count grows until voxel-first subsampling reaches `target`.
    raw = int(target * 1.6)
    while True:
        pts = []
        for (axis, val), area in zip(planes, areas):
            cnt = int(raw * area / total_area)
            o1, o2 = [a for a in range(3) if a != axis]
            p = np.empty((cnt, 3), np.float32)
            p[:, axis] = val
            p[:, o1] = rng.random(cnt, dtype=np.float32) * ext[o1]
            p[:, o2] = rng.random(cnt, dtype=np.float32) * ext[o2]
            pts.append(p)
        for lo, hi in boxes:
            a = (hi[0] - lo[0]) * (hi[1] - lo[1]) + 2 * (hi[2] - lo[2]) * ((hi[0] - lo[0]) + (hi[1] - lo[1]))
            pts.append(_box_faces(lo, hi, int(raw * a / total_area), rng))
        xyz = np.concatenate(pts).astype(np.float32)
        xyz += rng.normal(0.0, noise, xyz.shape).astype(np.float32)
        xyz -= xyz.min(0)
        xyz = np.round(xyz * 1000.0) / 1000.0  # millimetre grid, as the reference rounds
        xyz = voxel_first(xyz.astype(np.float32), voxel)
        if len(xyz) >= target or raw > 20 * target:
            break
        raw = int(raw * 1.5)
    rng.shuffle(xyz)
    return np.ascontiguousarray(xyz[:target] if len(xyz) > target else xyz)


def lidar(seed: int = SEED, rings: int = 64, azimuths: int = 2048, voxel: float = 0.05,
          max_range: float = 50.0, drop: float = 0.1, n_cyl: int = 60, n_box: int = 40,
          noise: float = 0.02, dedup: bool = False) -> np.ndarray:
    """Ray-cast spinning-LiDAR scan (sensor at the origin, ground at z=-1.7 m).

    Ground plane, vertical cylinders (poles, trunks), boxes (cars, buildings)
    and a ring of facades between 40 and 48 m catch the rays, so nearly every
    ray returns; 10% of the returns are dropped at random.  Density falls
    with range as 1/r^2.  Not voxel-deduplicated by default: a scan keeps
    several points per 5 cm voxel in the near field, as real scans do."""
    rng = np.random.default_rng(seed)
    elev = np.deg2rad(np.linspace(-24.8, 2.0, rings))
    az = np.linspace(0.0, 2 * np.pi, azimuths, endpoint=False)
    E, A = np.meshgrid(elev, az, indexing="ij")
    d = np.stack([np.cos(E) * np.cos(A), np.cos(E) * np.sin(A), np.sin(E)], -1).reshape(-1, 3)
    t = np.full(d.shape[0], np.inf)
    # ground plane z = -1.7
    down = d[:, 2] < -1e-6
    t[down] = -1.7 / d[down, 2]
    # vertical cylinders
    r_c = rng.uniform(4.0, 45.0, n_cyl)
    a_c = rng.uniform(0, 2 * np.pi, n_cyl)
    cx, cy = r_c * np.cos(a_c), r_c * np.sin(a_c)
    rad = rng.uniform(0.15, 0.8, n_cyl)
    top = rng.uniform(0.5, 8.0, n_cyl) - 1.7
    for i in range(n_cyl):
        a = d[:, 0] ** 2 + d[:, 1] ** 2
        b = -2 * (d[:, 0] * cx[i] + d[:, 1] * cy[i])
        c = cx[i] ** 2 + cy[i] ** 2 - rad[i] ** 2
        disc = b * b - 4 * a * c
        ok = (disc > 0) & (a > 1e-12)
        tt = np.where(ok, (-b - np.sqrt(np.maximum(disc, 0))) / (2 * np.maximum(a, 1e-12)), np.inf)
        z = tt * d[:, 2]
        hit = ok & (tt > 0) & (z >= -1.7) & (z <= top[i])
        t = np.where(hit & (tt < t), tt, t)
    # boxes (buildings / cars), slab test
    r_b = rng.uniform(6.0, 48.0, n_box)
    a_b = rng.uniform(0, 2 * np.pi, n_box)
    bx, by = r_b * np.cos(a_b), r_b * np.sin(a_b)
    sx, sy = rng.uniform(1.0, 8.0, n_box), rng.uniform(1.0, 8.0, n_box)
    sz = rng.uniform(1.0, 10.0, n_box)
    inv = 1.0 / np.where(np.abs(d) < 1e-12, 1e-12, d)
    for i in range(n_box):
        lo = np.array([bx[i] - sx[i] / 2, by[i] - sy[i] / 2, -1.7])
        hi = np.array([bx[i] + sx[i] / 2, by[i] + sy[i] / 2, -1.7 + sz[i]])
        t1 = lo * inv
        t2 = hi * inv
        tmin = np.minimum(t1, t2).max(1)
        tmax = np.maximum(t1, t2).min(1)
        hit = (tmax >= np.maximum(tmin, 0)) & (tmin > 0)
        t = np.where(hit & (tmin < t), tmin, t)
    # facades: an inside-out cylinder of radius 40..48 m per azimuth sector
    sectors = 24
    sec = (np.arctan2(d[:, 1], d[:, 0]) % (2 * np.pi)) / (2 * np.pi) * sectors
    wall_r = rng.uniform(40.0, 48.0, sectors)[sec.astype(np.int64) % sectors]
    wall_top = rng.uniform(4.0, 20.0, sectors)[sec.astype(np.int64) % sectors] - 1.7
    horiz = np.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2)
    tw = wall_r / np.maximum(horiz, 1e-12)
    zw = tw * d[:, 2]
    hit = (zw >= -1.7) & (zw <= wall_top)
    t = np.where(hit & (tw < t), tw, t)
    keep = np.isfinite(t) & (t <= max_range)
    keep &= rng.random(keep.shape[0]) >= drop
    t = t + rng.normal(0.0, noise, t.shape)
    xyz = (d[keep] * t[keep, None]).astype(np.float32)
    if dedup:
        xyz = voxel_first(xyz, voxel)
    return np.ascontiguousarray(xyz)


def crop(xyz: np.ndarray, count: int, rng) -> np.ndarray:
    """`count` points nearest to a random point (the reference's crop)."""
    if len(xyz) <= count:
        return xyz
    c = xyz[rng.integers(len(xyz))]
    order = np.argsort(((xyz - c) ** 2).sum(1), kind="stable")
    return np.ascontiguousarray(xyz[np.sort(order[:count])])


@dataclass
class Batch:
    xyz: np.ndarray       # f32 [N,3], clouds concatenated
    offsets: np.ndarray   # int64 [B], cumulative ends
    counts: np.ndarray    # int64 [B]
    kinds: list           # "room" / "lidar" per cloud
    voxel: float


def draw_counts(n_clouds=16, lo=20000, hi=200000, seed=SEED, total=1_500_000, tol=0.03):
    """Log-uniform cloud sizes.  The first seed >= `seed` whose draw totals
    within `tol` of `total` is used (the configuration names ~1.5M points)."""
    s = seed
    while True:
        rng = np.random.default_rng(s)
        counts = np.exp(rng.uniform(np.log(lo), np.log(hi), n_clouds)).astype(np.int64)
        if abs(counts.sum() - total) <= tol * total:
            return counts, s
        s += 1


def uneven_batch(n_clouds: int = 16, lo: int = 20000, hi: int = 200000, seed: int = SEED,
                 voxel: float = 0.05, total: int = 1_500_000, cache: bool = True) -> Batch:
    """C4: clouds with log-uniform sizes, alternating room-like / LiDAR-like.

    Cached in the temp directory (keyed by the arguments), since generating
    the ray-cast scans takes several seconds."""
    import hashlib
    import os
    import tempfile
    tag = hashlib.sha1(repr(("v2", n_clouds, lo, hi, seed, voxel, total)).encode()).hexdigest()[:12]
    path = os.path.join(tempfile.gettempdir(), f"fknn_uneven_batch_{tag}.npz")
    if cache and os.path.exists(path):
        z = np.load(path, allow_pickle=False)
        return Batch(xyz=z["xyz"], offsets=z["offsets"], counts=z["counts"],
                     kinds=[str(k) for k in z["kinds"]], voxel=float(z["voxel"]))
    batch = _uneven_batch(n_clouds, lo, hi, seed, voxel, total)
    if cache:
        tmp = path + f".{os.getpid()}.npz"
        np.savez(tmp, xyz=batch.xyz, offsets=batch.offsets, counts=batch.counts,
                 kinds=np.array(batch.kinds), voxel=np.float64(batch.voxel))
        os.replace(tmp, path)
    return batch


def _uneven_batch(n_clouds, lo, hi, seed, voxel, total) -> Batch:
    counts, seed = draw_counts(n_clouds, lo, hi, seed, total)
    rng = np.random.default_rng(seed)
    clouds, kinds = [], []
    for i, target in enumerate(counts):
        if i % 2 == 0:
            # scale the room so it holds enough 5 cm voxels
            scale = max(1.0, (target / 60000.0) ** 0.5)
            pts = room(seed=seed + 101 * i, target=int(target), voxel=voxel,
                       dims=(6.0 * scale, 8.0 * scale, 3.0))
            kinds.append("room")
        else:
            # voxel-first at the grid voxel, as the reference prepares its
            # LiDAR frames (scripts/prepare_semantickitti_pack.py:39-43,84);
            # enough rays that the deduplicated scan reaches the target size
            rings, az = next(((r, a) for r, a, cap in ((64, 2048, 70000), (128, 2048, 110000),
                                                       (128, 4096, 150000)) if target <= cap),
                             (256, 4096))
            pts = lidar(seed=seed + 101 * i, rings=rings, azimuths=az, voxel=voxel, dedup=True)
            kinds.append("lidar")
        pts = crop(pts, int(target), rng)
        clouds.append(pts.astype(np.float32))
    counts = np.array([len(c) for c in clouds], np.int64)
    return Batch(xyz=np.ascontiguousarray(np.concatenate(clouds)), offsets=np.cumsum(counts),
                 counts=counts, kinds=kinds, voxel=voxel)


def first_clouds(batch: Batch, count: int) -> Batch:
    """The first `count` clouds of a batch (smaller cases for profiling)."""
    end = int(batch.offsets[count - 1])
    return Batch(xyz=np.ascontiguousarray(batch.xyz[:end]), offsets=batch.offsets[:count].copy(),
                 counts=batch.counts[:count].copy(), kinds=batch.kinds[:count],
                 voxel=batch.voxel)


def backward_weights(n: int, k: int, seed: int = SEED) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal((n, k)).astype(np.float32)


# Grid voxel per configuration (num_down = 2, i.e. alpha = 4, unless stated).
C1_VOXEL = 0.0197
C2_VOXEL = 0.04
C3_VOXEL = 0.05
C4_VOXEL = 0.05
