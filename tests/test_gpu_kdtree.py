"""GPU parity of the k-d tree build, kNN and r-near (needs a B200).

Everything goes through the public drop-in API, which calls the C ABI.  The
expected answers come from the reference (golden fixtures) and from the CPU
oracle, which breaks distance ties by point index as the GPU does and
therefore must agree bit for bit.
"""
import math
import os

import numpy as np
import pytest

from _util import compare_knn, dist2

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["f32_uniform", "f64_uniform", "f32_nan_dups", "f32_grid", "f64_aniso"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.mark.parametrize("name", CASES)
def test_build_is_the_reference_tree(gpu, name):
    g = load(name)
    t = gpu.kdtree._build(g["points"])
    assert t.n_valid == len(g["reverse"])
    assert np.array_equal(t.reverse_indices(), g["reverse"])
    assert np.array_equal(t.ref_nodes(), g["nodes"])


@pytest.mark.parametrize("name", CASES)
def test_queries_match_reference(gpu, name):
    g = load(name)
    P, Q, k = g["points"], g["queries"], int(g["k"])
    t = gpu.kdtree._build(P)
    idx, cnt = gpu.kdtree.knn(t, Q, k)
    assert compare_knn(idx, cnt, g["knn_idx"], g["knn_cnt"], P, Q, k)[0] == 0
    idx, cnt = gpu.kdtree.knn(t, Q, k, dmax=float(g["knn_r_dmax"]))
    assert compare_knn(idx, cnt, g["knn_r_idx"], g["knn_r_cnt"], P, Q, k)[0] == 0
    rows = gpu.kdtree._query(t, Q, k=k)
    assert len(rows) == len(Q) and all(r.dtype == np.int32 for r in rows)
    assert all(np.array_equal(r, idx_row[:len(r)]) for r, idx_row in zip(rows, gpu.kdtree.knn(t, Q, k)[0]))
    sq = g["self_q"]
    sidx, scnt = gpu.kdtree.knn(t, sq, k)
    assert np.array_equal(scnt, g["self_cnt"])
    ok = scnt > 0
    Qs = P[np.where(ok, sq, 0)]
    assert compare_knn(sidx[ok], scnt[ok], g["self_idx"][ok], g["self_cnt"][ok], P, Qs[ok], k)[0] == 0
    off, out = gpu.kdtree.rnear(t, Q, float(g["rnear_r"]))
    assert np.array_equal(off, g["rnear_off"]) and np.array_equal(out, g["rnear_idx"])
    off, out = gpu.kdtree.rnear(t, sq, float(g["rnear_r"]))
    assert np.array_equal(off, g["rself_off"]) and np.array_equal(out, g["rself_idx"])
    rows = gpu.kdtree._query(t, sq, k=None, dmax=float(g["rnear_r"]))
    assert np.array_equal(np.concatenate(rows), g["rself_idx"])


def _tie_clouds():
    """Inputs full of exact distance ties (as in tests/test_oracle.py)."""
    import os as _os
    g = lambda n: dict(np.load(_os.path.join(GOLDEN, f"{n}.npz")))["points"]  # noqa: E731
    rng = np.random.default_rng(12)
    return {
        "f32_grid": g("f32_grid"),
        "f32_nan_dups": g("f32_nan_dups"),
        "identical": np.full((300, 3), 0.25, np.float32),
        "int16_grid": rng.integers(0, 6, (3000, 3)).astype(np.int16),
        "f64_lattice": np.stack(np.meshgrid(*[np.arange(10.0)] * 3), -1).reshape(-1, 3) * 0.5,
    }


@pytest.mark.parametrize("case", list(_tie_clouds()))
def test_knn_ties_broken_by_point_index(gpu, port, case):
    # at every exact distance tie the result is the k smallest
    # (dist2, point index) pairs, identical to the oracle: point, self and
    # all-points queries, every top-k capacity class and the device heaps
    # (k > 64), with packet walks and per-lane walks
    from pptk_b200 import _native as N
    P = _tie_clouds()[case]
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    rng = np.random.default_rng(14)
    qf = np.float64 if P.dtype == np.float64 else np.float32
    # index queries address rows 0 .. num_points()-1 (the valid count), as
    # in the reference
    sel = np.sort(rng.choice(t.n_valid, min(t.n_valid, 400), replace=False)).astype(np.int32)
    Q = P[rng.choice(len(P), min(len(P), 400), replace=False)].astype(qf)
    Q = Q[np.isfinite(Q.astype(np.float64)).all(1)]
    allq = np.arange(t.n_valid, dtype=np.int32)
    default = N.tune_get("lane_span")
    try:
        for span in (-1, 0):
            N.tune_set("lane_span", span)
            for k in (1, 4, 7, 16, 33, 64, 100):
                gi, gc = gpu.kdtree.knn(t, Q, k)
                oi, oc = o.knn(Q, k)
                assert np.array_equal(gc, oc) and np.array_equal(gi, oi), (span, k, "points")
                gi, gc = gpu.kdtree.knn(t, sel, k)
                oi, oc = o.knn_self(sel, k)
                assert np.array_equal(gc, oc) and np.array_equal(gi, oi), (span, k, "self")
                gi, gc = gpu.kdtree.knn(t, None, k)
                oi, oc = o.knn_self(allq, k)
                assert np.array_equal(gc, oc) and np.array_equal(gi, oi), (span, k, "all")
            gi, gc = gpu.kdtree.knn(t, Q, 16, dmax=1.0)
            oi, oc = o.knn(Q, 16, dmax=1.0)
            assert np.array_equal(gc, oc) and np.array_equal(gi, oi), (span, "dmax")
    finally:
        N.tune_set("lane_span", default)


def test_forest_and_multi_tree_ties_broken_by_point_index(gpu, port):
    # the same rule in ragged batches (one launch over many clouds) and in
    # multi-tree batches (one launch over several resident trees)
    import ctypes
    from pptk_b200 import _native as N
    from pptk_b200 import ragged
    rng = np.random.default_rng(15)
    clouds = [rng.integers(0, 5, (int(s), 3)).astype(np.float32) for s in (700, 40, 2500, 1, 900)]
    off = np.concatenate([[0], np.cumsum([len(c) for c in clouds])])
    f = ragged.Forest(np.concatenate(clouds), off)
    for k in (5, 16, 40):
        idx, cnt = f.knn(k)
        for c, cl in enumerate(clouds):
            oi, oc = port.PortTree(cl).knn_self(np.arange(len(cl), dtype=np.int32), k)
            gi = np.where(idx[off[c]:off[c + 1]] >= 0, idx[off[c]:off[c + 1]] - off[c], -1)
            assert np.array_equal(cnt[off[c]:off[c + 1]], oc) and np.array_equal(gi, oi), (k, c)
    trees = [gpu.kdtree._build(c) for c in clouds]
    qs = [c[rng.integers(0, len(c), min(len(c), 300))] + np.float32(0.5) for c in clouds]
    rows = np.concatenate([[0], np.cumsum([len(q) for q in qs])]).astype(np.int64)
    Q = np.ascontiguousarray(np.concatenate(qs))
    handles = (ctypes.c_void_p * len(trees))(*[t._h.value for t in trees])
    for k in (6, 20):
        idx = np.empty((len(Q), k), np.int32)
        cnt = np.empty(len(Q), np.int32)
        N.call("pptkg_multi_knn", handles, len(trees), N.ptr(Q), N.ptr(rows), 0, N.MEM_HOST, k, float("inf"),
               N.ptr(idx), N.ptr(cnt), None)
        for g, (cl, q) in enumerate(zip(clouds, qs)):
            oi, oc = port.PortTree(cl).knn(q, k)
            assert np.array_equal(idx[rows[g]:rows[g + 1]], oi) and np.array_equal(cnt[rows[g]:rows[g + 1]], oc)


@pytest.mark.parametrize("seed,dtype", [(0, np.float32), (1, np.float64)])
def test_knn_bit_exact_vs_oracle(gpu, port, seed, dtype):
    # config-1 shape: 200k uniform points, all points as queries, k = 16
    P = np.random.default_rng(seed).random((200_000, 3)).astype(dtype)
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    assert np.array_equal(t.reverse_indices(), o.reverse_indices())
    gi, gc = gpu.kdtree.knn(t, None, 16)
    oi, oc = o.knn_self(np.arange(len(P), dtype=np.int32), 16)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    q = P[::7] + dtype(1e-4)
    gi, gc = gpu.kdtree.knn(t, q, 16)
    oi, oc = o.knn(q, 16)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)


def test_bucket_size_never_changes_results(gpu):
    P = np.random.default_rng(3).random((50_000, 3), dtype=np.float32)
    t = gpu.kdtree._build(P)
    base = gpu.kdtree.knn(t, None, 12)
    r0 = gpu.kdtree.rnear(t, P[:3000], 0.03)
    for b in (1, 4, 8, 16, 64, 256):
        t.set_bucket(b)
        got = gpu.kdtree.knn(t, None, 12)
        assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1])
        r = gpu.kdtree.rnear(t, P[:3000], 0.03)
        assert np.array_equal(r[0], r0[0]) and np.array_equal(r[1], r0[1])


def test_rnear_matches_oracle_and_brute_force(gpu, port):
    rng = np.random.default_rng(4)
    P = rng.random((30_000, 3), dtype=np.float32)
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    q = rng.random((5000, 3), dtype=np.float32)
    r = float(np.float32(0.04))
    off, out = gpu.kdtree.rnear(t, q, r)
    ooff, oout = o.rnear(q, r)
    assert np.array_equal(off, ooff) and np.array_equal(out, oout)
    # brute force on a few rows: hits are exactly the points with dist2 < r^2
    r2 = np.float32(r) * np.float32(r)
    for i in range(0, 5000, 997):
        d = dist2(P, q[i:i + 1], np.arange(len(P))[None, :])[0]
        assert set(out[off[i]:off[i + 1]].tolist()) == set(np.flatnonzero(d < r2).tolist())
    # self form drops the query point
    sidx = np.arange(0, 30_000, 11, dtype=np.int32)
    off, out = gpu.kdtree.rnear(t, sidx, r)
    ooff, oout = o.rnear_self(sidx, r)
    assert np.array_equal(off, ooff) and np.array_equal(out, oout)


@pytest.mark.parametrize("dtype,dim", [(np.float32, 3), (np.float64, 3), (np.float32, 2), (np.float64, 4),
                                       (np.int16, 3)])
def test_rnear_warp_per_query_matches_packets_and_oracle(gpu, port, dtype, dim):
    # small batches give each query a whole warp (rnear_warp_queries); both
    # forms must return the oracle's hits in its order, for point and self
    # queries, radii from a few hits to most of the cloud (whole boxes taken
    # without distance tests) and the all-points form
    from pptk_b200 import _native as N
    rng = np.random.default_rng(21 + dim)
    scale = 1000.0 if np.issubdtype(dtype, np.integer) else 1.0
    P = (rng.random((40_000, dim)) * scale).astype(dtype)
    P[::997] = P[1::997]
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    q = (rng.random((1000, dim)) * scale).astype(np.float32 if np.issubdtype(dtype, np.integer) else dtype)
    sidx = np.arange(0, len(P), 41, dtype=np.int32)
    default = N.tune_get("rnear_warp_queries")
    try:
        for r in (0.03 * scale, 0.2 * scale, 0.6 * scale):
            rr = float(np.float32(r))
            ooff, oout = o.rnear(q, rr)
            soff, sout = o.rnear_self(sidx, rr)
            for wq in (0, 1 << 30):
                N.tune_set("rnear_warp_queries", wq)
                off, out = gpu.kdtree.rnear(t, q, r)
                assert np.array_equal(off, ooff) and np.array_equal(out, oout), (r, wq)
                off, out = gpu.kdtree.rnear(t, sidx, r)
                assert np.array_equal(off, soff) and np.array_equal(out, sout), (r, wq)
        r = 0.01 * scale
        aoff, aout = o.rnear_self(np.arange(len(P), dtype=np.int32), float(np.float32(r)))
        for wq in (0, 1 << 30):
            N.tune_set("rnear_warp_queries", wq)
            off, out = gpu.kdtree.rnear(t, None, r)
            assert np.array_equal(off, aoff) and np.array_equal(out, aout), wq
        # edge cases: an empty tree, one point, every point identical
        if dtype == np.float32 and dim == 3:
            for E in (np.zeros((0, 3), np.float32), np.array([[0.5, 0.5, 0.5]], np.float32),
                      np.ones((300, 3), np.float32)):
                te = gpu.kdtree._build(E)
                qe = np.array([[0.5, 0.5, 0.5], [1.0, 1.0, 1.0], [9.0, 9.0, 9.0]], np.float32)
                got = []
                for wq in (0, 1 << 30):
                    N.tune_set("rnear_warp_queries", wq)
                    got.append(gpu.kdtree.rnear(te, qe, 0.6))
                    if len(E):
                        got.append(gpu.kdtree.rnear(te, np.arange(len(E), dtype=np.int32), 0.6))
                half = len(got) // 2
                for a, b in zip(got[:half], got[half:]):
                    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                if len(E):
                    oe = port.PortTree(E)
                    ooff, oout = oe.rnear(qe, float(np.float32(0.6)))
                    assert np.array_equal(got[0][0], ooff) and np.array_equal(got[0][1], oout)
                else:
                    assert (got[0][0] == 0).all() and len(got[0][1]) == 0
    finally:
        N.tune_set("rnear_warp_queries", default)


def test_edge_cases(gpu, port):
    kd = gpu.kdtree
    # empty input
    t = kd._build(np.zeros((0, 3), np.float32))
    assert t.n_valid == 0
    idx, cnt = kd.knn(t, np.zeros((4, 3), np.float32), 3)
    assert (cnt == 0).all() and (idx == -1).all()
    assert kd._query(t, None, k=2) == []
    # a single point, fewer points than k, k larger than a leaf
    P = np.array([[0.5, 0.5, 0.5]], np.float32)
    t = kd._build(P)
    assert [r.tolist() for r in kd._query(t, np.array([[0, 0, 0]], np.float32), k=5)] == [[0]]
    assert [r.tolist() for r in kd._query(t, None, k=5)] == [[]]
    P = np.random.default_rng(8).random((37, 3), dtype=np.float32)
    t = kd._build(P)
    o = port.PortTree(P)
    gi, gc = kd.knn(t, None, 50)
    oi, oc = o.knn_self(np.arange(37, dtype=np.int32), 50)
    assert np.array_equal(gi, oi) and np.array_equal(gc, oc) and (gc == 36).all()
    # all points identical: one leaf of every point, ties everywhere
    P = np.ones((500, 3), np.float64)
    t = kd._build(P)
    gi, gc = kd.knn(t, None, 7)
    oi, oc = port.PortTree(P).knn_self(np.arange(500, dtype=np.int32), 7)
    assert np.array_equal(gi, oi) and np.array_equal(gc, oc)
    # dmax = 0 finds nothing; NaN rows are dropped and answer nothing
    P = np.random.default_rng(9).random((1000, 3), dtype=np.float32)
    P[::10] = np.nan
    t = kd._build(P)
    assert t.n_valid == 900
    idx, cnt = kd.knn(t, P[1:50], 4, dmax=0.0)
    assert (cnt == 0).all()
    idx, cnt = kd.knn(t, np.arange(0, 100, dtype=np.int32), 4)
    assert (cnt[::10] == 0).all() and (cnt[1::10] == 4).all()
    gi, gc = kd.knn(t, None, 5)  # rows 0 .. num_points()-1, as the reference
    assert gi.shape == (900, 5)
    oi, oc = port.PortTree(P).knn_self(np.arange(900, dtype=np.int32), 5)
    assert np.array_equal(gi, oi) and np.array_equal(gc, oc)


def test_query_argument_errors(gpu):
    kd = gpu.kdtree
    P = np.random.default_rng(10).random((100, 3))
    t = kd._build(P)
    with pytest.raises(ValueError):
        kd._query(t, np.zeros((0, 2)), k=1)  # wrong dim
    with pytest.raises(ValueError):
        kd._query(t, np.zeros((0, 3)), k="a")
    with pytest.raises(ValueError):
        kd._query(t, np.zeros((0, 3)), dmax="a")
    with pytest.raises(ValueError):
        kd._query(t, P[:2], k=0)
    with pytest.raises(ValueError):
        kd._query(t, P[:2], dmax=-1.0)
    with pytest.raises(ValueError):
        kd._query(t, P[:2], k=None)  # k=None needs a finite dmax
    with pytest.raises(RuntimeError):
        kd._query(t, [0, 100], k=1)
    with pytest.raises(ValueError):
        kd._query(t, np.zeros(7, bool), k=1)
    with pytest.raises(NotImplementedError):
        kd._query(t, slice(0, 3), k=1)
    with pytest.raises(TypeError):
        kd._query("not a tree", P[:2], k=1)
    with pytest.raises(TypeError):
        kd._query(t, "abc", k=1)
    # negative indices wrap; masks select
    a = kd._query(t, [-1, 0], k=3)
    b = kd._query(t, [99, 0], k=3)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    m = np.zeros(100, bool)
    m[[5, 7]] = True
    c = kd._query(t, m, k=3)
    d = kd._query(t, [5, 7], k=3)
    assert all(np.array_equal(x, y) for x, y in zip(c, d))
    # dmax is rounded through float32, as the reference does
    r = 0.1 + 1e-12
    e = kd._query(t, P[:5], k=None, dmax=r)
    f = kd._query(t, P[:5], k=None, dmax=float(np.float32(r)))
    assert all(np.array_equal(x, y) for x, y in zip(e, f))


def test_torch_cuda_inputs_stay_on_device(gpu):
    import torch
    P = torch.rand(20_000, 3, device="cuda")
    t = gpu.kdtree._build(P)
    idx, cnt = gpu.kdtree.knn(t, P[:1000], 8)
    assert idx.is_cuda and idx.shape == (1000, 8)
    ref_idx, _ = gpu.kdtree.knn(gpu.kdtree._build(P.cpu().numpy()), P[:1000].cpu().numpy(), 8)
    assert np.array_equal(idx.cpu().numpy(), ref_idx)


def test_scene_properties_at_scale(gpu, port):
    # 2M-point lidar-like scene: full-size properties plus sampled exact rows
    from pptk_b200 import synth
    P = synth.lidar_scene(2_000_000, seed=2)
    t = gpu.kdtree._build(P)
    idx, cnt = gpu.kdtree.knn(t, None, 32)
    assert (cnt == 32).all()
    rows = np.arange(len(P))
    assert not (idx == rows[:, None]).any()  # self excluded
    d = dist2(P, P[:200_000], idx[:200_000])
    assert (np.diff(d, axis=1) >= 0).all()  # ascending distance
    o = port.PortTree(P)
    assert np.array_equal(t.reverse_indices(), o.reverse_indices())
    sample = np.random.default_rng(0).choice(len(P), 20_000, replace=False).astype(np.int32)
    oi, oc = o.knn_self(sample, 32)
    assert np.array_equal(idx[sample], oi)
    off, out = gpu.kdtree.rnear(t, sample, 0.5)
    ooff, oout = o.rnear_self(sample, 0.5)
    assert np.array_equal(off, ooff) and np.array_equal(out, oout)


@pytest.mark.parametrize("dim", [2, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_2d_and_4d_trees_match_oracle(gpu, port, dim, dtype):
    rng = np.random.default_rng(10 + dim)
    P = rng.random((40_000, dim)).astype(dtype)
    P[::997] = P[1::997]  # a few duplicate points (distance ties)
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    assert np.array_equal(t.reverse_indices(), o.reverse_indices())
    gi, gc = gpu.kdtree.knn(t, None, 9)
    oi, oc = o.knn_self(np.arange(len(P), dtype=np.int32), 9)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    q = rng.random((3000, dim)).astype(dtype)
    gi, gc = gpu.kdtree.knn(t, q, 9, dmax=0.05)
    oi, oc = o.knn(q, 9, dmax=float(np.float32(0.05)))
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    r = 0.03 if dim == 2 else 0.12
    off, out = gpu.kdtree.rnear(t, q, r)
    ooff, oout = o.rnear(q, float(np.float32(r)))
    assert np.array_equal(off, ooff) and np.array_equal(out, oout)
    sidx = np.arange(0, len(P), 13, dtype=np.int32)
    off, out = gpu.kdtree.rnear(t, sidx, r)
    ooff, oout = o.rnear_self(sidx, float(np.float32(r)))
    assert np.array_equal(off, ooff) and np.array_equal(out, oout)
    # the list form of _query
    rows = gpu.kdtree._query(t, q[:50], k=4)
    ei, _ = o.knn(q[:50], 4)
    assert all(np.array_equal(a, b) for a, b in zip(rows, ei))


INT_TYPES = [np.int8, np.uint8, np.int16, np.uint16, np.int32, np.uint32, np.int64, np.uint64]


@pytest.mark.parametrize("dtype", INT_TYPES)
@pytest.mark.parametrize("dim", [2, 3])
def test_integer_trees_match_oracle(gpu, port, dtype, dim):
    # integer trees: built in their own type (midpoints and widths in C++
    # integer arithmetic, wrapping where the reference's does), queried in
    # float32; coordinates span the whole type so widths overflow
    info = np.iinfo(dtype)
    rng = np.random.default_rng(20 + dim)
    P = rng.integers(info.min, info.max, (12_000, dim), dtype=dtype, endpoint=True)
    P[:3000] = (P[:3000] // 64) * 3  # a dense clump with duplicates
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    assert t.dtype == np.dtype(dtype)
    assert np.array_equal(t.reverse_indices(), o.reverse_indices())
    assert np.array_equal(t.ref_nodes(), o.nodes())
    gi, gc = gpu.kdtree.knn(t, None, 6)
    oi, oc = o.knn_self(np.arange(len(P), dtype=np.int32), 6)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    q = P[rng.integers(0, len(P), 2000)].astype(np.float32) + np.float32(1.5)
    gi, gc = gpu.kdtree.knn(t, q, 6)
    oi, oc = o.knn(q, 6)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    r = float(np.float32(max(2.0, (float(info.max) - float(info.min)) / 4096)))
    off, out = gpu.kdtree.rnear(t, q[:500], r)
    ooff, oout = o.rnear(q[:500], r)
    assert np.array_equal(off, ooff) and np.array_equal(out, oout)
    # integer query arrays go through float32, one conversion per coordinate
    qi = P[:300]
    gi, gc = gpu.kdtree.knn(t, qi, 4)
    oi, oc = o.knn(qi.astype(np.float32), 4)
    assert np.array_equal(gi, oi)
    # re-cutting the traversal hierarchy keeps every answer
    t.set_bucket(16)
    gi2, _ = gpu.kdtree.knn(t, qi, 4)
    assert np.array_equal(gi2, gi)
    # normals are defined for float32 / float64 points only
    import ctypes
    from pptk_b200 import _native as N
    ev = np.empty((2, 3), np.float32)
    with pytest.raises(TypeError):
        N.call("pptkg_tree_normals", t._h, None, 2, N.MEM_HOST, 4, ctypes.c_float(np.inf), 1, 0, N.ptr(ev), None,
               None, None)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_large_k_matches_oracle(gpu, port, dtype):
    # k above the register lists' capacity (64): device-memory heaps
    rng = np.random.default_rng(30)
    P = rng.random((30_000, 3)).astype(dtype)
    P[::211] = P[1::211]  # duplicates (distance ties)
    t = gpu.kdtree._build(P)
    o = port.PortTree(P)
    for k in (65, 100, 257):
        gi, gc = gpu.kdtree.knn(t, None, k)
        oi, oc = o.knn_self(np.arange(len(P), dtype=np.int32), k)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi), k
    q = rng.random((4000, 3)).astype(dtype)
    gi, gc = gpu.kdtree.knn(t, q, 130, dmax=0.1)
    oi, oc = o.knn(q, 130, dmax=float(np.float32(0.1)))
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    assert (gc < 130).any() and (gc == 130).any()  # dmax cuts some lists short
    rows = gpu.kdtree._query(t, q[:20], k=200)
    ei, _ = o.knn(q[:20], 200)
    assert all(np.array_equal(a, b) for a, b in zip(rows, ei))
