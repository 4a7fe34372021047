"""Seeded synthetic point clouds for the benchmark workloads.

No dataset ships with the reference and none is needed: every workload is
generated from a fixed seed, so the same arrays come out on every machine.

* ``uniform_cube``   -- n float32 points uniform in [0, 1)^3.
* ``lidar_scene``    -- a lidar-like street scene: a ground plane over
  200 x 200 m with Gaussian height noise, 500 axis-aligned boxes (1-10 m
  sides) and 300 vertical cylinders (r 0.2-1 m, h 2-8 m) sampled on their
  surfaces, with point density falling as 1/d^2 from a sensor at the origin
  (d clamped to >= 1 m); 70% ground, 20% boxes, 10% cylinders.
* ``planar_patches`` -- float64 precision stress: thin 10 x 10 m planar
  patches with random orientations and normal-direction noise, translated
  by 1e5 m in x and y, plus uniform outliers.
* ``ragged_clouds``  -- many independent clouds of log-uniform sizes, each a
  union of Gaussian blobs and a noisy plane, concatenated with CSR offsets.
"""
import math

import numpy as np


def uniform_cube(n, seed=0, dtype=np.float32):
    return np.random.default_rng(seed).random((n, 3), dtype=np.float32).astype(dtype, copy=False)


def _ground(rng, n, half=100.0, sigma=0.01):
    """n points on the square [-half, half]^2 with density ~ 1/max(1, d)^2."""
    # angle marginal: w(theta) ~ 1/2 + ln R(theta), R = distance to the square's edge
    out = np.empty((0, 2))
    while out.shape[0] < n:
        need = int((n - out.shape[0]) * 1.3) + 1024
        th = rng.uniform(-math.pi, math.pi, need)
        R = half / np.maximum(np.abs(np.cos(th)), np.abs(np.sin(th)))
        w = 0.5 + np.log(R)
        keep = rng.random(need) * (0.5 + math.log(half * math.sqrt(2.0))) < w
        th, R = th[keep], R[keep]
        # radius: density ~ r on [0, 1) (weight 1/2), ~ 1/r on [1, R) (weight ln R)
        u = rng.random(th.shape[0])
        inner = u * (0.5 + np.log(R)) < 0.5
        r = np.where(inner, np.sqrt(rng.random(th.shape[0])), np.exp(rng.random(th.shape[0]) * np.log(R)))
        out = np.concatenate([out, np.stack([r * np.cos(th), r * np.sin(th)], 1)])
    xy = out[:n]
    z = rng.normal(0.0, sigma, n)
    return np.concatenate([xy, z[:, None]], 1)


def _boxes(rng, n, count=500, half=100.0):
    c = rng.uniform(-half, half, (count, 2))
    s = rng.uniform(1.0, 10.0, (count, 3))
    faces_area = np.stack([s[:, 0] * s[:, 1], s[:, 0] * s[:, 2], s[:, 0] * s[:, 2],
                           s[:, 1] * s[:, 2], s[:, 1] * s[:, 2]], 1)  # top, +-y sides, +-x sides
    area = faces_area.sum(1)
    d = np.maximum(1.0, np.hypot(c[:, 0], c[:, 1]))
    w = area / d ** 2
    per = rng.multinomial(n, w / w.sum())
    obj = np.repeat(np.arange(count), per)
    fa = faces_area[obj]
    face = (rng.random(n)[:, None] * fa.sum(1, keepdims=True) < np.cumsum(fa, 1)).argmax(1)
    u, v = rng.random(n), rng.random(n)
    sx, sy, sz = s[obj, 0], s[obj, 1], s[obj, 2]
    x = np.where(face == 0, (u - .5) * sx, np.where(face <= 2, (u - .5) * sx, np.where(face == 3, sx / 2, -sx / 2)))
    y = np.where(face == 0, (v - .5) * sy, np.where(face == 1, sy / 2, np.where(face == 2, -sy / 2, (u - .5) * sy)))
    z = np.where(face == 0, sz, v * sz)
    return np.stack([x + c[obj, 0], y + c[obj, 1], z], 1)


def _cylinders(rng, n, count=300, half=100.0):
    c = rng.uniform(-half, half, (count, 2))
    rad = rng.uniform(0.2, 1.0, count)
    h = rng.uniform(2.0, 8.0, count)
    area = 2 * math.pi * rad * h + math.pi * rad ** 2
    d = np.maximum(1.0, np.hypot(c[:, 0], c[:, 1]))
    w = area / d ** 2
    per = rng.multinomial(n, w / w.sum())
    obj = np.repeat(np.arange(count), per)
    side = rng.random(n) * area[obj] < 2 * math.pi * rad[obj] * h[obj]
    th = rng.uniform(0, 2 * math.pi, n)
    rr = np.where(side, rad[obj], rad[obj] * np.sqrt(rng.random(n)))
    z = np.where(side, rng.random(n) * h[obj], h[obj])
    return np.stack([c[obj, 0] + rr * np.cos(th), c[obj, 1] + rr * np.sin(th), z], 1)


def lidar_scene(n, seed=2):
    """float32 (n, 3) lidar-like scene (see module docstring)."""
    rng = np.random.default_rng(seed)
    ng = int(round(0.7 * n))
    nb = int(round(0.2 * n))
    nc = n - ng - nb
    pts = np.concatenate([_ground(rng, ng), _boxes(rng, nb), _cylinders(rng, nc)])
    perm = rng.permutation(n)
    return np.ascontiguousarray(pts[perm], dtype=np.float32)


def planar_patches(n, seed=3, count=200, size=10.0, sigma=1e-4, offset=1e5, outliers=0.05):
    """float64 (n, 3) precision-stress cloud and the true patch normal of
    every point (NaN for outliers)."""
    rng = np.random.default_rng(seed)
    n_out = int(round(outliers * n))
    n_in = n - n_out
    nrm = rng.normal(size=(count, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    a = np.cross(nrm, np.where(np.abs(nrm[:, :1]) < 0.9, [[1.0, 0, 0]], [[0, 1.0, 0]]))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = np.cross(nrm, a)
    cen = rng.uniform([0, 0, 0], [400, 400, 50], (count, 3))
    obj = rng.integers(0, count, n_in)
    u = rng.uniform(-size / 2, size / 2, n_in)
    v = rng.uniform(-size / 2, size / 2, n_in)
    e = rng.normal(0.0, sigma, n_in)
    p = cen[obj] + u[:, None] * a[obj] + v[:, None] * b[obj] + e[:, None] * nrm[obj]
    lo, hi = p.min(0), p.max(0)
    q = rng.uniform(lo, hi, (n_out, 3))
    pts = np.concatenate([p, q])
    tn = np.concatenate([nrm[obj], np.full((n_out, 3), np.nan)])
    perm = rng.permutation(n)
    pts = pts[perm]
    pts[:, 0] += offset
    pts[:, 1] += offset
    return np.ascontiguousarray(pts), tn[perm]


def ragged_sizes(count=4096, lo=1000, hi=200000, seed=4):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)


def ragged_clouds(count=4096, lo=1000, hi=200000, seed=4):
    """(points float32 (sum, 3), offsets int64 (count + 1))."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)
    off = np.concatenate([[0], np.cumsum(sizes)])
    out = np.empty((int(off[-1]), 3), np.float32)
    for i in range(count):
        s = int(sizes[i])
        nb = int(rng.integers(1, 6))
        n_plane = s // 3
        n_blob = s - n_plane
        cen = rng.uniform(-5, 5, (nb, 3))
        sig = rng.uniform(0.05, 0.5, nb)
        which = rng.integers(0, nb, n_blob)
        blobs = cen[which] + rng.normal(size=(n_blob, 3)) * sig[which, None]
        nrm = rng.normal(size=3)
        nrm /= np.linalg.norm(nrm)
        a = np.cross(nrm, [1.0, 0, 0] if abs(nrm[0]) < 0.9 else [0, 1.0, 0])
        a /= np.linalg.norm(a)
        b = np.cross(nrm, a)
        uv = rng.uniform(-5, 5, (n_plane, 2))
        plane = uv[:, :1] * a + uv[:, 1:] * b + rng.normal(0, 0.01, (n_plane, 1)) * nrm
        out[off[i]:off[i + 1]] = np.concatenate([blobs, plane])
    return out, off


def request_mix(n_points, per_kind, seed=10, lo=1000, hi=1_000_000):
    """Seeded request stream over an n-point scene: alternating kNN and
    normal requests with query counts log-uniform in [lo, hi], until each
    kind totals `per_kind` queries.  Returns [(kind, rows)] with rows the
    int32 scene rows a request asks about (kNN requests query those points'
    coordinates, normal requests those rows)."""
    rng = np.random.default_rng(seed)
    left = {"knn": int(per_kind), "normals": int(per_kind)}
    out = []
    kind = "knn"
    while left["knn"] > 0 or left["normals"] > 0:
        if left[kind] > 0:
            m = int(np.exp(rng.uniform(math.log(lo), math.log(hi))))
            m = max(1, min(m, left[kind]))
            out.append((kind, rng.integers(0, n_points, m).astype(np.int32)))
            left[kind] -= m
        kind = "normals" if kind == "knn" else "knn"
    return out
