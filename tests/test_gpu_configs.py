"""Parity at the full sizes of the benchmark configurations (needs a B200).

* 20M-point lidar scene (float32): kNN k=32 for every point, bit-exact
  against the oracle on 20k sampled rows, with size-independent properties
  checked on every row; r-near r=0.5 m counts (20k rows) and hit lists
  (2k rows) exact against the oracle; normals k=16 on the FP32 path against
  the FP64 oracle on 20k rows.
* 10M-point float64 planar patches offset by 1e5 m: normals k=24 on the
  FP32 path against the FP64 oracle (p99 <= 1e-4 rad, |dot| >= 1 - 1e-6
  where the eigen-gap defines a normal) and on the FP64 path to 1e-5
  relative per eigenvalue.
* 4,096 ragged clouds (158M points): one forest build, kNN k=16 and normals
  for every point; sampled clouds exact against the oracle, properties on
  every row.
* The 64-tree serving mix at a tenth of its point count (64 lidar scenes of
  50k-400k points): a burst of kNN (k 8..64), r-near (r 0.1..1 m), normal
  and build requests through the server, every answer equal to the direct
  single-tree call on the same tree.

The oracle runs on the host over the same seeded inputs; neighbourhoods for
the FP64 normal oracle come from the oracle's own kNN (ties by point index).
"""
import numpy as np
import pytest

from _util import angle_error

pytestmark = pytest.mark.gpu
DOT_TOL = 1e-6
GAP_EXCLUDE = 1e-4


def _fp64_check(port, P, rows, nb, ev32, label, p99_max=1e-4):
    """FP32-path normals of `rows` against the FP64 oracle over the oracle's
    neighbourhoods nb: |dot| >= 1 - 1e-6 where the relative eigen-gap is at
    least 1e-4, p99 angular error <= p99_max over all rows."""
    w, V, _ = port.normals_fp64(P, nb)
    gap = (w[:, 1] - w[:, 0]) / np.maximum(np.abs(w[:, 2]), 1e-300)
    ok = gap >= GAP_EXCLUDE
    dots = np.abs((ev32.astype(np.float64) * V[:, 0, :]).sum(1))
    assert (dots[ok] >= 1 - DOT_TOL).all(), (label, np.sort(dots[ok])[:5])
    ang = angle_error(ev32, V[:, 0, :])
    assert np.percentile(ang, 99) <= p99_max, (label, np.percentile(ang, 99))
    assert (~ok).sum() < 0.01 * len(rows), label
    return w


def test_scene_20M(gpu, port):
    import torch
    from pptk_b200 import synth
    P = synth.lidar_scene(20_000_000, seed=2)
    n = len(P)
    dev = torch.from_numpy(P).cuda()
    t = gpu.kdtree._build(dev)
    o = port.PortTree(P)
    assert np.array_equal(t.reverse_indices(), o.reverse_indices())
    rows = np.sort(np.random.default_rng(20).choice(n, 20_000, replace=False)).astype(np.int32)
    # kNN k=32 for every point (self queries), results left on the device
    from pptk_b200 import _native as N
    idx = torch.empty((n, 32), dtype=torch.int32, device="cuda")
    cnt = torch.empty((n,), dtype=torch.int32, device="cuda")
    N.call("pptkg_knn_self", t._h, None, n, N.MEM_DEVICE, 32, float("inf"), N.ptr(idx), N.ptr(cnt),
           N.torch_stream())
    assert bool((cnt == 32).all())
    ar = torch.arange(n, device="cuda", dtype=torch.int32)[:, None]
    assert not bool((idx == ar).any())  # the query point is excluded
    assert bool(((idx >= 0) & (idx < n)).all())
    # ascending distance on every row (computed on the device in float32,
    # the reference's arithmetic: per-axis difference, squared, summed in
    # axis order)
    for lo in range(0, n, 2_000_000):
        nb = dev[idx[lo:lo + 2_000_000].long()]
        d = nb - dev[lo:lo + 2_000_000, None, :]
        d2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
        assert bool((d2[:, 1:] >= d2[:, :-1]).all())
    oi, oc = o.knn_self(rows, 32)
    assert np.array_equal(idx[torch.from_numpy(rows).cuda().long()].cpu().numpy(), oi)
    del idx, cnt
    # r-near r = 0.5 m: counts for 20k rows, hit lists for 2k
    off, _ = gpu.kdtree.rnear(t, rows, 0.5)
    ooff, _ = o.rnear_self(rows, 0.5)
    assert np.array_equal(off, ooff)
    few = rows[::10]
    off, hits = gpu.kdtree.rnear(t, few, 0.5)
    ooff, ohits = o.rnear_self(few, 0.5)
    assert np.array_equal(off, ooff) and np.array_equal(hits, ohits)
    # normals k=16, FP32 path, against the FP64 oracle
    ev = gpu.estimate_normals(dev, 16, np.inf, subsample=rows, verbose=False).cpu().numpy()
    nbr, ncnt = o.knn(P[rows], 16)
    assert (ncnt == 16).all()
    _fp64_check(port, P, rows, nbr, ev, "scene k=16")


def test_planar_patches_10M_f64(gpu, port):
    import torch
    from pptk_b200 import synth
    P, _ = synth.planar_patches(10_000_000, seed=3)
    dev = torch.from_numpy(P).cuda()
    rows = np.sort(np.random.default_rng(21).choice(len(P), 20_000, replace=False)).astype(np.int32)
    n32, w32, s32 = gpu.estimate_normals(dev, 24, np.inf, subsample=rows, precision="fp32", output_eigenvalues=True,
                                         output_neighborhood_sizes=True, verbose=False)
    n64, w64, s64 = gpu.estimate_normals(dev, 24, np.inf, subsample=rows, precision="fp64",
                                         output_eigenvalues=True, output_all_eigenvectors=True,
                                         output_neighborhood_sizes=True, verbose=False)
    o = port.PortTree(P)
    nb, nc = o.knn(P[rows], 24)
    assert np.array_equal(s32.cpu().numpy(), nc) and np.array_equal(s64.cpu().numpy(), nc)
    w = _fp64_check(port, P, rows, nb, n32.cpu().numpy(), "patches fp32 path")
    # FP64 path: normals and every eigenvalue to 1e-5 relative
    W64 = w64.cpu().numpy()
    assert (np.abs(W64 - w) <= 1e-5 * np.abs(w)).all()
    _fp64_check(port, P, rows, nb, n64.cpu().numpy()[:, 0, :], "patches fp64 path", p99_max=1e-6)


def test_ragged_4096_clouds(gpu, port):
    import torch
    from pptk_b200 import ragged, synth
    P, off = synth.ragged_clouds(4096, seed=4)
    sizes = np.diff(off)
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    idx, cnt = f.knn(16)
    ev = f.normals(16)
    # every row: counts and neighbours inside the own cloud
    want = torch.from_numpy(np.minimum(16, sizes - 1).repeat(sizes).astype(np.int32)).cuda()
    assert torch.equal(cnt, want)
    cloud_of = torch.from_numpy(np.repeat(np.arange(4096), sizes).astype(np.int64)).cuda()
    first = idx[:, 0].long()
    assert bool((cloud_of[first] == cloud_of).all())
    assert bool(torch.isfinite(ev).all())
    # sampled clouds: kNN exact against the oracle, normals against FP64
    pick = sorted({int(np.argmin(sizes)), int(np.argmax(sizes)), 0, 1000, 2047, 4095})
    for c in pick:
        cl = P[off[c]:off[c + 1]]
        tc = port.PortTree(cl)
        oi, oc = tc.knn_self(np.arange(len(cl), dtype=np.int32), 16)
        gi = idx[off[c]:off[c + 1]].cpu().numpy()
        assert np.array_equal(np.where(gi >= 0, gi - off[c], -1), oi), c
        rows = np.arange(len(cl), dtype=np.int32)[:: max(1, len(cl) // 5000)]
        nb, _ = tc.knn(cl[rows], 16)
        _fp64_check(port, cl, rows, nb, ev[off[c]:off[c + 1]].cpu().numpy()[rows], f"cloud {c}")


def test_rnear_normals_match_fp64_oracle(gpu, port):
    # r-near neighbourhoods (k = -1): every point within r, itself included;
    # sizes exact, normals against the FP64 oracle to |dot| >= 1 - 1e-6
    P = np.random.default_rng(22).random((40_000, 3)).astype(np.float32)
    P[:, 2] *= 0.2
    r = 0.04
    ev, ew, sz = gpu.estimate_normals(P, -1, r, output_eigenvalues=True, output_all_eigenvectors=True,
                                      output_neighborhood_sizes=True, verbose=False)
    o = port.PortTree(P)
    ooff, ohits = o.rnear(P, float(np.float32(r)))
    assert np.array_equal(sz, np.diff(ooff))
    X = P[ohits].astype(np.float64)
    cnt = np.diff(ooff)
    keep = cnt >= 5
    seg = np.repeat(np.arange(len(P)), cnt)
    mean = np.add.reduceat(X, ooff[:-1], axis=0) / np.maximum(cnt, 1)[:, None]
    Y = X - mean[seg]
    C = np.stack([np.add.reduceat(Y[:, i] * Y[:, j], ooff[:-1]) for i in range(3) for j in range(3)], 1)
    C = C.reshape(-1, 3, 3) / np.maximum(cnt, 1)[:, None, None]
    w, V = np.linalg.eigh(C[keep])
    gap = (w[:, 1] - w[:, 0]) / np.maximum(np.abs(w[:, 2]), 1e-300)
    ok = gap >= GAP_EXCLUDE
    dots = np.abs((ev[keep, 0, :].astype(np.float64) * V[:, :, 0]).sum(1))
    assert (dots[ok] >= 1 - DOT_TOL).all(), np.sort(dots[ok])[:5]
    assert ok.sum() > 0.95 * keep.sum()


def test_multitree_mix_shape(gpu):
    import threading
    from pptk_b200 import estimate_normals, kdtree, serving, synth
    rng = np.random.default_rng(17)
    sizes = rng.integers(50_000, 400_001, 64)
    clouds = [synth.lidar_scene(int(n), seed=300 + i) for i, n in enumerate(sizes)]
    srv = serving.Server(budget_bytes=40e9, slots=3)
    ids = [f.result(timeout=300) for f in [srv.build(c) for c in clouds]]
    reqs = []
    for _ in range(240):
        u = rng.random()
        g = int(rng.integers(0, 64))
        m = int(np.exp(rng.uniform(np.log(1e3), np.log(5e4))))
        if u < 0.05:
            reqs.append(("build", g, synth.lidar_scene(int(rng.integers(20_000, 200_000)), seed=int(rng.integers(1e6)))))
        elif u < 0.45:
            q = clouds[g][rng.integers(0, len(clouds[g]), m)] + np.float32(5e-3)
            reqs.append(("knn", g, (q, int(rng.integers(8, 65)))))
        elif u < 0.60:
            q = clouds[g][rng.integers(0, len(clouds[g]), min(m, 2_000))]
            reqs.append(("rnear", g, (q, float(np.float32(rng.uniform(0.1, 1.0))))))
        else:
            reqs.append(("normals", g, rng.integers(0, len(clouds[g]), m).astype(np.int32)))

    def submit(kind, g, a):
        if kind == "knn":
            return srv.knn(ids[g], a[0], k=a[1])
        if kind == "rnear":
            return srv.rnear(ids[g], a[0], a[1])
        if kind == "normals":
            return srv.normals(ids[g], a, k=16)
        return srv.build(a)

    futs = [submit(*r) for r in reqs]
    results = [f.result(timeout=600) for f in futs]
    for (kind, g, a), got in zip(reqs, results):
        tree = srv.trees[ids[g]]
        if kind == "knn":
            direct, cnt = kdtree.knn(tree, a[0], a[1])
            assert np.array_equal(got[0], direct) and np.array_equal(got[1], cnt), (g, a[1])
        elif kind == "rnear":
            off, hits = kdtree.rnear(tree, a[0], a[1])
            assert np.array_equal(got[0], off) and np.array_equal(got[1], hits), g
        elif kind == "normals":
            direct = estimate_normals(clouds[g], 16, np.inf, subsample=a, verbose=False)
            assert np.array_equal(np.nan_to_num(got, nan=-9.0), np.nan_to_num(direct, nan=-9.0)), g
        else:
            q = a[:300] + np.float32(1e-3)
            direct, _ = kdtree.knn(kdtree._build(a), q, 8)
            assert np.array_equal(srv.knn(got, q, k=8).result(timeout=120)[0], direct)
    st = srv.stats()
    assert st["knn"]["requests"] + st["rnear"]["requests"] + st["normals"]["requests"] >= 200
    srv.close()
