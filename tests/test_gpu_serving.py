"""Multi-tree batches and the serving loop on the GPU: every answer is the
same alone and in the mix (bit for bit)."""
import ctypes
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def trees_and_queries(gpu, seed=0):
    rng = np.random.default_rng(seed)
    clouds = [rng.random((int(s), 3), dtype=np.float32) * rng.uniform(1, 10)
              for s in (50_000, 3, 20_000, 120_000)]
    trees = [gpu.kdtree._build(c) for c in clouds]
    qs = [c[rng.integers(0, len(c), int(m))] + np.float32(1e-3) for c, m in zip(clouds, (4000, 2, 0, 9000))]
    return clouds, trees, qs


def test_multi_tree_knn_equals_single_tree(gpu):
    from pptk_b200 import _native as N
    clouds, trees, qs = trees_and_queries(gpu)
    rows = np.concatenate([[0], np.cumsum([len(q) for q in qs])]).astype(np.int64)
    Q = np.ascontiguousarray(np.concatenate(qs))
    m, k = len(Q), 12
    idx = np.empty((m, k), np.int32)
    cnt = np.empty(m, np.int32)
    handles = (ctypes.c_void_p * len(trees))(*[t._h.value for t in trees])
    N.call("pptkg_multi_knn", handles, len(trees), N.ptr(Q), N.ptr(rows), 0, N.MEM_HOST, k, float("inf"),
           N.ptr(idx), N.ptr(cnt), None)
    for g, (t, q) in enumerate(zip(trees, qs)):
        if len(q) == 0:
            continue
        si, sc = gpu.kdtree.knn(t, q, k)
        assert np.array_equal(idx[rows[g]:rows[g + 1]], si) and np.array_equal(cnt[rows[g]:rows[g + 1]], sc)


def test_multi_tree_normals_equal_single_tree(gpu):
    from pptk_b200 import _native as N
    clouds, trees, _ = trees_and_queries(gpu, seed=1)
    rng = np.random.default_rng(2)
    ids = [rng.integers(0, len(c), min(len(c), 5000)).astype(np.int32) for c in clouds]
    rows = np.concatenate([[0], np.cumsum([len(i) for i in ids])]).astype(np.int64)
    I = np.ascontiguousarray(np.concatenate(ids))
    ev = np.empty((len(I), 3), np.float32)
    handles = (ctypes.c_void_p * len(trees))(*[t._h.value for t in trees])
    N.call("pptkg_multi_normals", handles, len(trees), N.ptr(I), N.ptr(rows), N.MEM_HOST, 10,
           ctypes.c_float(np.inf), 1, 0, N.ptr(ev), None, None, None)
    for g, (t, ix) in enumerate(zip(trees, ids)):
        alone = np.empty((len(ix), 3), np.float32)
        N.call("pptkg_tree_normals", t._h, N.ptr(ix), len(ix), N.MEM_HOST, 10, ctypes.c_float(np.inf), 1, 0,
               N.ptr(alone), None, None, None)
        assert np.array_equal(ev[rows[g]:rows[g + 1]], alone)


def _np(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


def test_server_answers_are_the_same_alone_and_in_the_mix(gpu):
    import torch
    from pptk_b200 import serving
    rng = np.random.default_rng(3)
    clouds = [rng.random((int(s), 3), dtype=np.float32) for s in (80_000, 30_000, 150_000)]
    srv = serving.Server(budget_bytes=8e9, slots=3)
    ids = [f.result(timeout=120) for f in [srv.build(c) for c in clouds]]
    reqs = []
    for i in range(40):
        g = int(rng.integers(0, 3))
        if i % 2:
            q = clouds[g][rng.integers(0, len(clouds[g]), int(rng.integers(1, 20_000)))] + np.float32(2e-3)
            reqs.append(("knn", g, q))
        else:
            ix = rng.integers(0, len(clouds[g]), int(rng.integers(1, 20_000))).astype(np.int32)
            reqs.append(("normals", g, ix))
    # every third request passes CUDA tensors (and gets CUDA tensors back)
    reqs = [(kind, g, torch.from_numpy(a).cuda() if j % 3 == 0 else a) for j, (kind, g, a) in enumerate(reqs)]
    results = [None] * len(reqs)

    def client(lo, hi):
        for j in range(lo, hi):
            kind, g, a = reqs[j]
            f = srv.knn(ids[g], a, k=8) if kind == "knn" else srv.normals(ids[g], a, k=8)
            results[j] = f.result(timeout=120)

    threads = [threading.Thread(target=client, args=(j, j + 10)) for j in range(0, 40, 10)]
    [t.start() for t in threads]
    [t.join() for t in threads]
    st = srv.stats()
    assert st["knn"]["requests"] == 20 and st["normals"]["requests"] == 20
    # alone: the same requests one at a time
    for j, ((kind, g, a), got) in enumerate(zip(reqs, results)):
        f = srv.knn(ids[g], a, k=8) if kind == "knn" else srv.normals(ids[g], a, k=8)
        alone = f.result(timeout=120)
        on_device = j % 3 == 0
        if kind == "knn":
            assert all(torch.is_tensor(x) == on_device for x in got)
            assert np.array_equal(_np(got[0]), _np(alone[0])) and np.array_equal(_np(got[1]), _np(alone[1]))
            direct, _ = gpu.kdtree.knn(srv.trees[ids[g]], _np(a), 8)
            assert np.array_equal(_np(got[0]), direct)
        else:
            assert torch.is_tensor(got) == on_device
            assert np.array_equal(_np(got), _np(alone))
    srv.close()


def test_multi_tree_normals_rejects_an_index_outside_its_tree(gpu):
    from pptk_b200 import _native as N
    clouds, trees, _ = trees_and_queries(gpu, seed=4)
    ids = [np.arange(min(len(c), 100), dtype=np.int32) for c in clouds]
    ids[1] = np.array([0, 1, 3], np.int32)  # the second tree holds 3 points: row 3 is outside
    rows = np.concatenate([[0], np.cumsum([len(i) for i in ids])]).astype(np.int64)
    I = np.ascontiguousarray(np.concatenate(ids))
    ev = np.empty((len(I), 3), np.float32)
    handles = (ctypes.c_void_p * len(trees))(*[t._h.value for t in trees])
    with pytest.raises(RuntimeError, match="outside"):
        N.call("pptkg_multi_normals", handles, len(trees), N.ptr(I), N.ptr(rows), N.MEM_HOST, 10,
               ctypes.c_float(np.inf), 1, 0, N.ptr(ev), None, None, None)
    # the library stays usable after the error
    ids[1] = np.array([0, 1, 2], np.int32)
    I = np.ascontiguousarray(np.concatenate(ids))
    N.call("pptkg_multi_normals", handles, len(trees), N.ptr(I), N.ptr(rows), N.MEM_HOST, 10,
           ctypes.c_float(np.inf), 1, 0, N.ptr(ev), None, None, None)
    assert np.isfinite(ev).all()


def test_server_merges_knn_requests_of_one_k_class(gpu):
    from pptk_b200 import serving
    rng = np.random.default_rng(8)
    cloud = rng.random((200_000, 3), dtype=np.float32)
    srv = serving.Server(budget_bytes=8e9, slots=1)
    tid = srv.build(cloud).result(timeout=120)
    blocker = srv.normals(tid, None, k=32)  # keeps the only slot busy while the others queue
    qs = {5: cloud[:3000] + np.float32(1e-3), 7: cloud[5000:6000] - np.float32(1e-3), 20: cloud[9000:9100]}
    futs = {k: srv.knn(tid, q, k=k) for k, q in qs.items()}
    blocker.result(timeout=120)
    tree = srv.trees[tid]
    for k, q in qs.items():
        idx, cnt = futs[k].result(timeout=120)
        di, dc = gpu.kdtree.knn(tree, q, k)
        assert np.array_equal(idx, di) and np.array_equal(cnt, dc), k
    srv.close()
