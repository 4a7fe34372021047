"""Scheduling logic of the serving loop, on a fake engine (CPU only)."""
import math
import threading
import time

import numpy as np
import pytest

from pptk_b200 import serving


class FakeTree:
    def __init__(self, pts):
        self.pts = np.asarray(pts, np.float64)
        self.n = len(pts)
        self.dtype = np.float64


class FakeEngine:
    """Brute-force CPU stand-in with a controllable delay per batch."""

    def __init__(self, delay=0.0):
        self.delay = delay
        self.batches = []
        self.lock = threading.Lock()

    def stream(self, high_priority=False):
        return object()

    def build(self, points, maxleafsize, emptysplit, stream):
        time.sleep(self.delay)
        return FakeTree(points)

    def knn_batch(self, trees, queries, k, dmax, stream, host=False):
        with self.lock:
            self.batches.append(("knn", len(trees), k))
        time.sleep(self.delay)
        out = []
        for t, q in zip(trees, queries):
            d = ((np.asarray(q)[:, None, :] - t.pts[None]) ** 2).sum(-1)
            idx = np.argsort(d, axis=1, kind="stable")[:, :k].astype(np.int32)
            out.append((idx, np.full(len(q), min(k, t.n), np.int32)))
        return out

    def normals_batch(self, trees, indices, k, r, precision, stream, host=False):
        with self.lock:
            self.batches.append(("normals", len(trees)))
        return [np.zeros((t.n if i is None else len(i), 3)) for t, i in zip(trees, indices)]

    def rnear(self, tree, queries, dmax, stream):
        return ([0], [])

    def synchronize(self, stream):
        pass


def test_results_and_batching():
    eng = FakeEngine(delay=0.05)
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng)
    rng = np.random.default_rng(0)
    pts = [rng.random((200, 3)) for _ in range(3)]
    ids = [srv.build(p).result(timeout=10) for p in pts]
    qs = [rng.random((int(rng.integers(1, 50)), 3)) for _ in range(12)]
    futs = [srv.knn(ids[i % 3], q, k=5) for i, q in enumerate(qs)]
    for i, (q, f) in enumerate(zip(qs, futs)):
        idx, cnt = f.result(timeout=10)
        d = ((q[:, None, :] - pts[i % 3][None]) ** 2).sum(-1)
        assert np.array_equal(idx, np.argsort(d, axis=1, kind="stable")[:, :5])
    # the requests submitted while the first batch ran were folded together
    knn_batches = [b for b in eng.batches if b[0] == "knn"]
    assert len(knn_batches) < len(qs)
    st = srv.stats()
    assert st["knn"]["requests"] == len(qs) and st["knn"]["p99_s"] >= st["knn"]["p50_s"]
    srv.close()


def test_budget_admission_and_errors():
    eng = FakeEngine()
    srv = serving.Server(budget_bytes=200 * (serving.TREE_BYTES_PER_POINT + serving.BUILD_SCRATCH_PER_POINT),
                         slots=2, engine=eng)
    with pytest.raises(MemoryError):
        srv.build(np.zeros((10_000, 3))).result(timeout=10)
    tid = srv.build(np.random.rand(100, 3)).result(timeout=10)
    with pytest.raises(KeyError):
        srv.knn(tid + 99, np.zeros((2, 3)), k=1).result(timeout=10)
    # committed tree bytes stay reserved until the tree is dropped
    assert srv._committed == pytest.approx(100 * serving.TREE_BYTES_PER_POINT)
    srv.drop(tid)
    assert srv._committed == pytest.approx(0.0)
    srv.close()


def test_fifo_order_is_kept_across_kinds():
    eng = FakeEngine(delay=0.01)
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng)
    tid = srv.build(np.random.rand(50, 3)).result(timeout=10)
    f1 = srv.knn(tid, np.random.rand(3, 3), k=2)
    f2 = srv.build(np.random.rand(40, 3))
    f3 = srv.normals(tid, None, k=4)
    f1.result(timeout=10), f2.result(timeout=10), f3.result(timeout=10)
    assert f3.result().shape == (50, 3)
    srv.close()


def test_knn_requests_of_one_k_class_share_a_launch():
    eng = FakeEngine(delay=0.05)
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng)
    rng = np.random.default_rng(1)
    pts = rng.random((300, 3))
    tid = srv.build(pts).result(timeout=10)
    blocker = srv.knn(tid, rng.random((4, 3)), k=3)  # holds the only slot for a while
    qs = {5: rng.random((6, 3)), 7: rng.random((5, 3)), 20: rng.random((3, 3))}
    futs = {k: srv.knn(tid, q, k=k) for k, q in qs.items()}
    blocker.result(timeout=10)
    for k, q in qs.items():
        idx, cnt = futs[k].result(timeout=10)
        d = ((q[:, None, :] - pts[None]) ** 2).sum(-1)
        assert idx.shape == (len(q), k)
        assert np.array_equal(idx, np.argsort(d, axis=1, kind="stable")[:, :k])
        assert (cnt == k).all()
    launches = [b for b in eng.batches if b[0] == "knn"][1:]
    # k = 5 and 7 (capacity class 8) ran as one k = 7 launch; k = 20 on its own
    assert sorted(b[2] for b in launches) == [7, 20]
    srv.close()
