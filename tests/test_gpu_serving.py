"""Multi-tree batches and the serving loop on the GPU: every answer is the
same alone and in the mix (bit for bit)."""
import ctypes
import threading
import time

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
    # kNN, normal, r-near and build requests of very different sizes, from
    # four client threads at once, against the same requests one at a time
    import torch
    from pptk_b200 import serving
    rng = np.random.default_rng(3)
    clouds = [rng.random((int(s), 3), dtype=np.float32) for s in (80_000, 30_000, 150_000)]
    srv = serving.Server(budget_bytes=8e9, slots=3, max_batch_queries=6_000, min_batch_queries=1_000,
                         small_batch=2_000)
    ids = [f.result(timeout=120) for f in [srv.build(c) for c in clouds]]
    reqs = []
    for i in range(48):
        g = int(rng.integers(0, 3))
        u = i % 6
        if u in (1, 3):
            q = clouds[g][rng.integers(0, len(clouds[g]), int(rng.integers(1, 20_000)))] + np.float32(2e-3)
            reqs.append(("knn", g, q))
        elif u in (0, 2):
            ix = rng.integers(0, len(clouds[g]), int(rng.integers(1, 20_000))).astype(np.int32)
            reqs.append(("normals", g, ix))
        elif u == 4:
            q = clouds[g][rng.integers(0, len(clouds[g]), int(rng.integers(1, 3_000)))]
            reqs.append(("rnear", g, q))
        else:
            reqs.append(("build", g, rng.random((int(rng.integers(1_000, 60_000)), 3), dtype=np.float32)))
    # every third request passes CUDA tensors (and gets CUDA tensors back)
    reqs = [(kind, g, torch.from_numpy(a).cuda() if j % 3 == 0 else a) for j, (kind, g, a) in enumerate(reqs)]
    results = [None] * len(reqs)

    def submit(kind, g, a):
        if kind == "knn":
            return srv.knn(ids[g], a, k=8)
        if kind == "normals":
            return srv.normals(ids[g], a, k=8)
        if kind == "rnear":
            return srv.rnear(ids[g], a, 0.03)
        return srv.build(a)

    def client(lo, hi):
        for j in range(lo, hi):
            results[j] = submit(*reqs[j]).result(timeout=120)

    threads = [threading.Thread(target=client, args=(j, j + 12)) for j in range(0, 48, 12)]
    [t.start() for t in threads]
    [t.join() for t in threads]
    st = srv.stats()
    assert st["knn"]["requests"] == 16 and st["normals"]["requests"] == 16 and st["rnear"]["requests"] == 8
    assert st["batches"] > 8
    # alone: the same requests one at a time
    for j, ((kind, g, a), got) in enumerate(zip(reqs, results)):
        alone = submit(kind, g, a).result(timeout=120)
        on_device = j % 3 == 0
        if kind == "knn":
            assert all(torch.is_tensor(x) == on_device for x in got)
            assert np.array_equal(_np(got[0]), _np(alone[0])) and np.array_equal(_np(got[1]), _np(alone[1]))
            direct, _ = gpu.kdtree.knn(srv.trees[ids[g]], _np(a), 8)
            assert np.array_equal(_np(got[0]), direct)
        elif kind == "normals":
            assert torch.is_tensor(got) == on_device
            assert np.array_equal(_np(got), _np(alone))
        elif kind == "rnear":
            off, hits = gpu.kdtree.rnear(srv.trees[ids[g]], _np(a), 0.03)
            for x in (got, alone):
                assert np.array_equal(_np(x[0]), off) and np.array_equal(_np(x[1]), hits)
        else:
            # a tree built in the mix answers like a tree built alone
            pts = _np(a)
            q = pts[:500] + np.float32(1e-3)
            direct, _ = gpu.kdtree.knn(gpu.kdtree._build(pts), q, 6)
            for tid in (got, alone):
                assert np.array_equal(srv.knn(tid, q, k=6).result(timeout=120)[0], direct)
    srv.close()


def test_server_batches_overlap_on_the_device(gpu):
    # three slots, requests sliced into several batches: CUDA events on the
    # slot streams show batches of different slots in flight on the device
    # at the same time
    import torch
    from pptk_b200 import serving
    rng = np.random.default_rng(9)
    cloud = rng.random((1_000_000, 3), dtype=np.float32)
    srv = serving.Server(budget_bytes=8e9, slots=3, max_batch_queries=400_000, min_batch_queries=100_000,
                         small_batch=1, trace=True)
    tid = srv.build(torch.from_numpy(cloud).cuda()).result(timeout=120)
    torch.cuda.synchronize()
    ref = torch.cuda.Event(enable_timing=True)
    ref.record()  # before every batch event below
    torch.cuda.synchronize()
    futs = [srv.normals(tid, torch.from_numpy(rng.integers(0, len(cloud), 1_200_000).astype(np.int32)).cuda(),
                        k=16) for _ in range(2)]
    futs.append(srv.knn(tid, torch.from_numpy(cloud[:1_200_000 // 2]).cuda(), k=16))
    [f.result(timeout=120) for f in futs]
    torch.cuda.synchronize()
    tr = [t for t in srv.trace if t[0] != ["build"]]
    assert len(tr) >= 6
    iv = [(ref.elapsed_time(t[2]), ref.elapsed_time(t[3])) for t in tr]
    overlaps = sum(1 for i in range(len(iv)) for j in range(i + 1, len(iv))
                   if iv[i][0] < iv[j][1] and iv[j][0] < iv[i][1])
    assert overlaps >= 2, iv
    srv.close()


def test_small_request_finishes_before_a_large_one_submitted_earlier(gpu):
    # a 1k-query request submitted behind a 10M-query request is answered
    # first: the large one runs in slices, the small one on the fast slot
    import torch
    from pptk_b200 import serving
    rng = np.random.default_rng(10)
    cloud = torch.from_numpy(rng.random((2_000_000, 3), dtype=np.float32)).cuda()
    srv = serving.Server(budget_bytes=16e9, slots=3)
    tid = srv.build(cloud).result(timeout=120)
    big_rows = torch.from_numpy(rng.integers(0, 2_000_000, 10_000_000).astype(np.int32)).cuda()
    small_q = cloud[:1000] + 1e-3
    torch.cuda.synchronize()
    done = {}
    big = srv.normals(tid, big_rows, k=16)
    small = srv.knn(tid, small_q, k=16)
    big.add_done_callback(lambda f: done.setdefault("big", time.perf_counter()))
    small.add_done_callback(lambda f: done.setdefault("small", time.perf_counter()))
    small.result(timeout=120)
    big.result(timeout=120)
    assert done["small"] < done["big"]
    idx, _ = small.result()
    direct, _ = gpu.kdtree.knn(srv.trees[tid], small_q, 16)
    assert torch.equal(idx, direct)
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
