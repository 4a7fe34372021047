"""The CPU oracle, pinned against the reference (CPU only).

The restatement in oracle/port.cpp is checked against the golden fixtures
generated from the reference's own k-d tree (tests/golden/make_golden.py),
against the reference's known-answer tests, and -- when the reference harness
is built -- against the reference live on further inputs.
"""
import os

import numpy as np
import pytest

from _util import brute_knn, compare_knn

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["f32_uniform", "f64_uniform", "f32_nan_dups", "f32_grid", "f64_aniso"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.mark.parametrize("name", CASES)
def test_port_tree_matches_reference_golden(port, name):
    g = load(name)
    t = port.PortTree(g["points"])
    assert np.array_equal(t.reverse_indices(), g["reverse"])
    assert np.array_equal(t.nodes(), g["nodes"])


@pytest.mark.parametrize("name", CASES)
def test_port_queries_match_reference_golden(port, name):
    g = load(name)
    P, Q, k = g["points"], g["queries"], int(g["k"])
    t = port.PortTree(P)
    idx, cnt = t.knn(Q, k)
    mism, ties = compare_knn(idx, cnt, g["knn_idx"], g["knn_cnt"], P, Q, k)
    assert mism == 0
    idx, cnt = t.knn(Q, k, dmax=float(g["knn_r_dmax"]))
    mism, _ = compare_knn(idx, cnt, g["knn_r_idx"], g["knn_r_cnt"], P, Q, k)
    assert mism == 0
    # self queries: the query point is removed from its own result
    sq = g["self_q"]
    sidx, scnt = t.knn_self(sq, k)
    assert np.array_equal(scnt, g["self_cnt"])
    ok = scnt > 0
    Qs = np.where(ok[:, None], P[np.where(ok, sq, 0)], 0).astype(P.dtype)
    mism, _ = compare_knn(sidx[ok], scnt[ok], g["self_idx"][ok], g["self_cnt"][ok], P, Qs[ok], k)
    assert mism == 0
    # r-near comes back in the reference's exact order
    off, out = t.rnear(Q, float(g["rnear_r"]))
    assert np.array_equal(off, g["rnear_off"]) and np.array_equal(out, g["rnear_idx"])
    off, out = t.rnear_self(sq, float(g["rnear_r"]))
    assert np.array_equal(off, g["rself_off"]) and np.array_equal(out, g["rself_idx"])


def _tie_clouds():
    """Inputs full of exact distance ties: the golden grid and duplicate
    sets, all-identical points, and integer grids."""
    rng = np.random.default_rng(12)
    yield "f32_grid", load("f32_grid")["points"]
    yield "f32_nan_dups", load("f32_nan_dups")["points"]
    yield "identical", np.full((300, 3), 0.25, np.float32)
    yield "int16_grid", rng.integers(0, 6, (3000, 3)).astype(np.int16)
    yield "uint8_grid2d", rng.integers(0, 9, (2500, 2)).astype(np.uint8)
    yield "f64_lattice", (np.stack(np.meshgrid(*[np.arange(10.0)] * 3), -1).reshape(-1, 3) * 0.5)


@pytest.mark.parametrize("case", [c for c, _ in _tie_clouds()])
def test_port_knn_breaks_ties_by_point_index(port, case):
    # the specified kNN answer: the k smallest (dist2, point index) pairs.
    # Exhaustive search defines it independently of any tree.
    P = dict(_tie_clouds())[case]
    t = port.PortTree(P)
    rng = np.random.default_rng(13)
    qf = np.float64 if P.dtype == np.float64 else np.float32
    sel = rng.choice(len(P), min(len(P), 150), replace=False)
    Q = P[sel].astype(qf)
    finite = np.isfinite(Q.astype(np.float64)).all(1)
    Q = Q[finite]
    for k, dmax in ((1, np.inf), (7, np.inf), (16, np.inf), (16, 1.0)):
        idx, cnt = t.knn(Q, k, dmax=dmax)
        bi, bc = brute_knn(P, Q, k, dmax)
        assert np.array_equal(cnt, bc) and np.array_equal(idx, bi), (case, k, dmax)
        sq = sel[finite].astype(np.int32)
        sidx, scnt = t.knn_self(sq, k, dmax=dmax)
        bi, bc = brute_knn(P, Q, k, dmax, exclude=sq)
        assert np.array_equal(scnt, bc) and np.array_equal(sidx, bi), (case, k, dmax)


def test_knearest_known_answer(port):
    # reference tests/test_points.py:299-308: 100 float64 points, 5 queries,
    # k=10, results equal to argsort of the squared distances, in order
    np.random.seed(0)
    P = np.random.rand(100, 3)
    Q = np.random.rand(5, 3)
    J = np.stack([np.argsort(((P - q) ** 2).sum(1))[:10] for q in Q])
    idx, cnt = port.PortTree(P).knn(Q, 10)
    assert (cnt == 10).all() and np.array_equal(idx, J)


def test_collinear_normals_known_answer(port):
    # reference tests/test_estimate_normals.py:38-138 on the restatement
    g = load("collinear_normals")
    ev, ew, sz = port.port_estimate_normals(g["points"], 4, 3.0, num_eigen=3)
    assert np.array_equal(sz, [3] + [4] * 8 + [3])
    assert np.allclose(ew[:, -1], [2.0 / 3] + [5.0 / 4] * 8 + [2.0 / 3])
    assert np.allclose(ev[:, -1, :], [[1.0, 0.0, 0.0]] * 10)
    assert np.array_equal(sz, g["sizes"])
    assert np.allclose(ew, g["evals"]) and np.allclose(np.abs(ev[:, -1]), np.abs(g["evecs"][:, -1]))
    # subsample by mask and by indices with a negative one
    s = [0, 3, 4, -1]
    ev2, ew2, sz2 = port.port_estimate_normals(g["points"], 4, 3.0, subsample=np.array([0, 3, 4, 9]), num_eigen=3)
    assert np.array_equal(sz2, np.asarray(sz)[s]) and np.allclose(ew2, ew[s])


def test_port_normals_agree_with_fp64_oracle(port):
    rng = np.random.default_rng(5)
    P = rng.random((4000, 3))
    ev, ew, sz, nb = port.port_estimate_normals(P, 12, np.inf, num_eigen=3, want_nbrs=True)
    w, V, _ = port.normals_fp64(P, nb)
    assert np.allclose(ew, w, rtol=1e-9, atol=1e-12)
    dots = np.abs((ev[:, 0, :] * V[:, 0, :]).sum(1))
    assert (dots > 1 - 1e-9).all()


def test_port_eigh3_matches_lapack(port):
    rng = np.random.default_rng(6)
    X = rng.normal(size=(500, 3, 3))
    A = X @ np.transpose(X, (0, 2, 1))
    w, V = port.port_eigh3(A)
    wl, Vl = np.linalg.eigh(A)
    assert np.allclose(w, wl, rtol=1e-10, atol=1e-10)
    assert (np.abs((V * Vl).sum(1)) > 1 - 1e-10).all()  # columns are eigenvectors


def _rank_pair_partition(vals, s):
    """The scan formulation used by the device builder: per pass, the j-th
    misplaced element of the left zone (ascending) swaps with the j-th
    misplaced element of the right zone (descending)."""
    a = list(range(len(vals)))
    v = lambda i: vals[a[i]]  # noqa: E731
    n = len(a)
    L1 = sum(1 for x in vals if x < s)
    L2 = sum(1 for x in vals if x <= s)
    for lo, Z, bad, good in ((0, L1, lambda x: x >= s, lambda x: x < s),
                             (L1, L2, lambda x: x > s, lambda x: x <= s)):
        bl = [i for i in range(lo, Z) if bad(v(i))]
        gr = [i for i in range(n - 1, Z - 1, -1) if good(v(i))]
        assert len(bl) == len(gr)
        for x, y in zip(bl, gr):
            a[x], a[y] = a[y], a[x]
    return a, L1, L2


def test_scan_partition_equals_two_cursor_partition(port):
    # the GPU builder's rank pairing must give the permutation of the
    # reference's converging-cursor passes; compared through whole trees
    rng = np.random.default_rng(7)
    for trial in range(200):
        n = int(rng.integers(1, 60))
        vals = rng.integers(0, 6, n).astype(np.float64)
        s = float(rng.integers(0, 6))
        perm, L1, L2 = _rank_pair_partition(list(vals), s)
        out = [vals[i] for i in perm]
        assert all(x < s for x in out[:L1]) and all(x == s for x in out[L1:L2]) and all(x > s for x in out[L2:])
        # against a direct restatement of the two cursor passes
        a = list(range(n))
        lo, hi = 0, n - 1
        for cond_l, cond_r in ((lambda x: x < s, lambda x: x >= s), (lambda x: x <= s, lambda x: x > s)):
            hi = n - 1
            while True:
                while lo <= hi and cond_l(vals[a[lo]]):
                    lo += 1
                while lo <= hi and cond_r(vals[a[hi]]):
                    hi -= 1
                if lo >= hi:
                    break
                a[lo], a[hi] = a[hi], a[lo]
                lo += 1
                hi -= 1
        assert a == perm


@pytest.mark.parametrize("dtype,dim", [(np.float32, 3), (np.float64, 2), (np.float32, 4), (np.int32, 3),
                                       (np.uint16, 2), (np.int64, 4)])
def test_port_matches_reference_live(ref, dtype, dim):
    rng = np.random.default_rng(11)
    if np.dtype(dtype).kind == "f":
        P = rng.normal(size=(6000, dim)).astype(dtype)
    else:
        P = rng.integers(0, 200, (6000, dim)).astype(dtype)
    a, b = ref.PortTree(P), ref.RefTree(P)
    assert np.array_equal(a.reverse_indices(), b.reverse_indices())
    assert np.array_equal(a.nodes(), b.nodes())
    q = P[:300].astype(np.float64) if np.dtype(dtype).kind != "f" else P[:300]
    oa = a.rnear(q, 3.0)
    ob = b.rnear(q, 3.0)
    assert np.array_equal(oa[0], ob[0]) and np.array_equal(oa[1], ob[1])
    # kNN: the same answers up to the reference's choice among tied points
    # (integer clouds are full of ties)
    qq = q.astype(np.float32) if np.dtype(dtype).kind != "f" else q
    ia, ca = a.knn(q, 9)
    ib, cb = b.knn(q, 9)
    assert compare_knn(ia, ca, ib, cb, P, qq, 9)[0] == 0
