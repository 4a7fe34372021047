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

    def rnear(self, tree, queries, dmax, stream, host=False):
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


def wait_started(eng, kind, count=1, timeout=10.0):
    """Waits until the engine has begun `count` batches of `kind`."""
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < timeout:
        with eng.lock:
            if sum(1 for b in eng.batches if b[0] == kind) >= count:
                return
        time.sleep(0.001)
    raise TimeoutError(kind)


class FailingEngine(FakeEngine):
    """Raises in the batches whose first request has the marked size, as an
    allocation refusal or a CUDA error of the native library would."""

    def __init__(self, fail_m, exc, delay=0.0):
        super().__init__(delay)
        self.fail_m = fail_m
        self.exc = exc

    def knn_batch(self, trees, queries, k, dmax, stream, host=False):
        if any(len(q) == self.fail_m for q in queries):
            with self.lock:
                self.batches.append(("knn-failed", len(trees), k))
            raise self.exc
        return super().knn_batch(trees, queries, k, dmax, stream, host)

    def normals_batch(self, trees, indices, k, r, precision, stream, host=False):
        if any(len(i) == self.fail_m for i in indices):
            raise self.exc
        return super().normals_batch(trees, indices, k, r, precision, stream, host)


@pytest.mark.parametrize("exc", [MemoryError("device allocation refused"),
                                 RuntimeError("CUDA error: an illegal memory access was encountered")])
def test_a_failing_batch_fails_only_its_requests(exc):
    eng = FailingEngine(fail_m=13, exc=exc, delay=0.02)
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng)
    rng = np.random.default_rng(2)
    pts = rng.random((100, 3))
    tid = srv.build(pts).result(timeout=10)
    blocker = srv.knn(tid, rng.random((4, 3)), k=2)  # holds the only slot while the next ones queue
    wait_started(eng, "knn")
    bad = [srv.knn(tid, rng.random((13, 3)), k=3), srv.normals(tid, np.arange(13, dtype=np.int32), k=4)]
    blocker.result(timeout=10)
    for f in bad:
        with pytest.raises(type(exc)):
            f.result(timeout=10)
    # the server keeps serving: later requests succeed
    q = rng.random((7, 3))
    idx, cnt = srv.knn(tid, q, k=3).result(timeout=10)
    d = ((q[:, None, :] - pts[None]) ** 2).sum(-1)
    assert np.array_equal(idx, np.argsort(d, axis=1, kind="stable")[:, :3])
    assert srv.normals(tid, np.arange(9, dtype=np.int32), k=4).result(timeout=10).shape == (9, 3)
    assert srv._committed == pytest.approx(100 * serving.TREE_BYTES_PER_POINT)
    srv.close()


def test_large_requests_are_answered_in_slices():
    # a request above the batch cap runs as several batches; its answer is
    # the same as in one piece
    eng = FakeEngine(delay=0.0)
    srv = serving.Server(budget_bytes=1e9, slots=2, engine=eng, max_batch_queries=64, min_batch_queries=1,
                         small_batch=16)
    rng = np.random.default_rng(3)
    pts = rng.random((500, 3))
    tid = srv.build(pts).result(timeout=10)
    q = rng.random((300, 3))
    idx, cnt = srv.knn(tid, q, k=4).result(timeout=10)
    d = ((q[:, None, :] - pts[None]) ** 2).sum(-1)
    assert np.array_equal(idx, np.argsort(d, axis=1, kind="stable")[:, :4]) and (cnt == 4).all()
    assert len([b for b in eng.batches if b[0] == "knn"]) >= 300 // 64
    ev = srv.normals(tid, None, k=4).result(timeout=10)
    assert ev.shape == (500, 3)
    srv.close()


def test_small_request_overtakes_a_large_one():
    # a small request submitted behind a large one is served by the fast
    # slot while the large one's slices run on the other
    eng = FakeEngine(delay=0.03)
    srv = serving.Server(budget_bytes=1e9, slots=2, engine=eng, max_batch_queries=100, min_batch_queries=1,
                         small_batch=50)
    rng = np.random.default_rng(4)
    tid = srv.build(rng.random((200, 3))).result(timeout=10)
    big = srv.knn(tid, rng.random((1000, 3)), k=2)
    time.sleep(0.01)
    small = srv.knn(tid, rng.random((5, 3)), k=2)
    small.result(timeout=10)
    assert not big.done()
    big.result(timeout=10)
    st = srv.stats()
    assert st["knn"]["requests"] == 2
    srv.close()


def test_cancelled_requests_never_run():
    eng = FakeEngine(delay=0.05)
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng)
    rng = np.random.default_rng(5)
    tid = srv.build(rng.random((100, 3))).result(timeout=10)
    blocker = srv.knn(tid, rng.random((3, 3)), k=2)
    wait_started(eng, "knn")
    doomed = srv.knn(tid, rng.random((11, 3)), k=2)
    kept = srv.knn(tid, rng.random((6, 3)), k=2)
    assert doomed.cancel()
    blocker.result(timeout=10)
    idx, _ = kept.result(timeout=10)
    assert idx.shape == (6, 2) and doomed.cancelled()
    with eng.lock:
        sizes = [b for b in eng.batches if b[0] == "knn"]
    assert len(sizes) == 2  # the blocker and the kept request; the cancelled one never ran
    srv.close()


def test_batch_cap_follows_the_measured_rate():
    eng = FakeEngine(delay=0.0)
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng, max_batch_queries=10_000_000,
                         min_batch_queries=1000, batch_ms=10.0)
    assert srv.batch_cap() == 10_000_000  # no rate measured yet: the upper bound
    srv._rate = 2e8
    assert srv.batch_cap() == 2_000_000
    srv._rate = 1e4
    assert srv.batch_cap() == 1000  # never below the lower bound
    srv.close()


def test_deferred_batches_fold_the_requests_that_arrive_during_a_batch():
    # while one normal-slot batch runs, the other normal slot waits for
    # min_batch_queries queued queries (or defer_ms) instead of starting a
    # small batch; the requests then run together
    eng = FakeEngine(delay=0.2)
    srv = serving.Server(budget_bytes=1e9, slots=3, fast_slots=1, engine=eng, small_batch=4,
                         min_batch_queries=100, defer_ms=5_000)
    rng = np.random.default_rng(6)
    pts = rng.random((100, 3))
    tid = srv.build(pts).result(timeout=10)
    blocker = srv.knn(tid, rng.random((10, 3)), k=2)
    wait_started(eng, "knn")
    qs = [rng.random((20, 3)) for _ in range(2)]
    futs = [srv.knn(tid, q, k=2) for q in qs]
    blocker.result(timeout=10)
    for q, f in zip(qs, futs):
        idx, _ = f.result(timeout=10)
        d = ((q[:, None, :] - pts[None]) ** 2).sum(-1)
        assert np.array_equal(idx, np.argsort(d, axis=1, kind="stable")[:, :2])
    with eng.lock:
        knn = [b for b in eng.batches if b[0] == "knn"]
    assert len(knn) == 2 and knn[1][1] == 2  # the blocker, then both requests in one launch
    srv.close()


def test_deferral_ends_after_defer_ms():
    eng = FakeEngine(delay=1.0)
    srv = serving.Server(budget_bytes=1e9, slots=3, fast_slots=1, engine=eng, small_batch=4,
                         min_batch_queries=100, defer_ms=50)
    rng = np.random.default_rng(7)
    tid = srv.build(rng.random((50, 3))).result(timeout=10)
    blocker = srv.knn(tid, rng.random((10, 3)), k=2)
    wait_started(eng, "knn")
    t0 = time.perf_counter()
    late = srv.knn(tid, rng.random((20, 3)), k=2)
    wait_started(eng, "knn", count=2, timeout=0.8)  # starts while the blocker still runs
    assert time.perf_counter() - t0 >= 0.04
    assert not blocker.done()
    late.result(timeout=10)
    srv.close()


class AsyncHostEngine(FakeEngine):
    """Host results that, like pinned copies on a stream, are only filled in
    when the stream is synchronised."""

    def __init__(self):
        super().__init__()
        self.pending = []

    def knn_batch(self, trees, queries, k, dmax, stream, host=False):
        out = super().knn_batch(trees, queries, k, dmax, stream, host)
        empty = []
        for idx, cnt in out:
            e_idx, e_cnt = np.zeros_like(idx), np.zeros_like(cnt)
            self.pending.append((e_idx, idx, e_cnt, cnt))
            empty.append((e_idx, e_cnt))
        return empty

    def synchronize(self, stream):
        with self.lock:
            for e_idx, idx, e_cnt, cnt in self.pending:
                e_idx[...] = idx
                e_cnt[...] = cnt
            self.pending = []


def test_knn_counts_of_a_merged_launch_wait_for_the_host_copies():
    # requests of one k class run at the class's largest k; each takes its
    # first k columns and its count capped at k -- only after the host
    # copies have landed
    eng = AsyncHostEngine()
    srv = serving.Server(budget_bytes=1e9, slots=1, engine=eng)
    rng = np.random.default_rng(8)
    pts = rng.random((300, 3))
    tid = srv.build(pts).result(timeout=10)
    blocker = srv.knn(tid, rng.random((3, 3)), k=8)
    wait_started(eng, "knn")
    qs = [rng.random((10, 3)) for _ in range(2)]
    futs = [srv.knn(tid, qs[0], k=5), srv.knn(tid, qs[1], k=7)]
    blocker.result(timeout=10)
    for q, f, k in zip(qs, futs, (5, 7)):
        idx, cnt = f.result(timeout=10)
        d = ((q[:, None, :] - pts[None]) ** 2).sum(-1)
        assert np.array_equal(idx, np.argsort(d, axis=1, kind="stable")[:, :k])
        assert (cnt == k).all()
    srv.close()
