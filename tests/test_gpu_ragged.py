"""Ragged batches (forests) on the GPU: every cloud's tree is the reference
tree for that cloud alone, and one forest query equals per-cloud queries."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_batch(seed=0, count=40, dtype=np.float32):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, 3000, count)
    sizes[3] = 0          # an empty cloud
    sizes[5] = 7          # smaller than a leaf
    sizes[7] = 9000       # above the per-CTA subtree size
    clouds = [rng.normal(size=(s, 3)).astype(dtype) * rng.uniform(0.1, 5.0) for s in sizes]
    clouds[9][::13] = np.nan  # dropped rows
    off = np.concatenate([[0], np.cumsum(sizes)])
    return np.concatenate(clouds), off, clouds


def test_forest_trees_are_the_reference_trees(gpu, port):
    from pptk_b200 import ragged
    P, off, clouds = small_batch()
    f = ragged.Forest(P, off)
    assert f.ncloud == len(clouds)
    rev = f.reverse_indices()
    for c, cl in enumerate(clouds):
        t = port.PortTree(cl)
        lo, hi = f.valid_offsets[c], f.valid_offsets[c + 1]
        assert np.array_equal(rev[lo:hi] - off[c], t.reverse_indices()), c
        assert np.array_equal(f.ref_nodes(c), t.nodes()), c


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_forest_queries_equal_per_cloud_queries(gpu, port, dtype):
    from pptk_b200 import ragged
    P, off, clouds = small_batch(seed=1, dtype=dtype)
    f = ragged.Forest(P, off)
    idx, cnt = f.knn(8)
    ev, ew, sz = f.normals(8, output_eigenvalues=True, output_neighborhood_sizes=True)
    for c, cl in enumerate(clouds):
        rows = slice(off[c], off[c + 1])
        if len(cl) == 0:
            continue
        t = port.PortTree(cl)
        nv = t.num_valid
        oi, oc = t.knn_self(np.arange(len(cl), dtype=np.int32), 8)
        gi = np.where(idx[rows] >= 0, idx[rows] - off[c], -1)
        assert np.array_equal(cnt[rows], oc) and np.array_equal(gi, oi), c
        # normals of the cloud alone through the drop-in API
        z = gpu.estimate_normals(cl, 8, np.inf, output_eigenvalues=True, output_neighborhood_sizes=True,
                                 verbose=False)
        assert np.array_equal(sz[rows], z[2]), c
        ok = np.isfinite(z[1])
        dots = np.abs((ev[rows][ok].astype(np.float64) * z[0][ok]).sum(1))
        assert (dots > 1 - 1e-6).all(), c
        assert nv == int((z[2] > 0).sum())


def test_forest_from_device_tensors(gpu):
    import torch
    from pptk_b200 import ragged
    P, off, clouds = small_batch(seed=2, count=12)
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    idx, cnt = f.knn(4)
    assert idx.is_cuda
    g = ragged.Forest(P, off)
    gi, gc = g.knn(4)
    assert np.array_equal(idx.cpu().numpy(), gi) and np.array_equal(cnt.cpu().numpy(), gc)


def test_ragged_config_shape_at_scale(gpu, port):
    # 256 clouds of the config-4 shape (log-uniform sizes, blobs + plane);
    # exact on sampled clouds, properties everywhere
    from pptk_b200 import ragged, synth
    P, off = synth.ragged_clouds(256, seed=4)
    f = ragged.Forest(P, off)
    idx, cnt = f.knn(16)
    assert (cnt == np.minimum(16, np.diff(off).repeat(np.diff(off)) - 1)).all()
    cloud_of = np.repeat(np.arange(256), np.diff(off))
    assert (cloud_of[idx[:, 0]] == cloud_of).all()  # neighbours stay in their cloud
    for c in (0, 17, 100, 255):
        cl = P[off[c]:off[c + 1]]
        oi, oc = port.PortTree(cl).knn_self(np.arange(len(cl), dtype=np.int32), 16)
        assert np.array_equal(idx[off[c]:off[c + 1]] - off[c], oi)


def test_captured_forest_queries_replay(gpu):
    import torch
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=5, count=20)
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    cap, (idx, cnt) = f.capture_knn(8)
    ref_i, ref_c = f.knn(8)
    for _ in range(2):
        idx.fill_(-7)
        cnt.fill_(-7)
        cap.replay()
        torch.cuda.synchronize()
        cap.check()
        assert torch.equal(idx, ref_i) and torch.equal(cnt, ref_c)
    capn, ev = f.capture_normals(8)
    ref_n = f.normals(8)
    ev.fill_(5.0)
    capn.replay()
    capn.check()
    assert torch.equal(torch.nan_to_num(ev, nan=-9.0), torch.nan_to_num(ref_n, nan=-9.0))


def test_builds_on_alternating_streams_agree(gpu):
    # forest builds take their scratch and tree arrays from a per-stream
    # cache of freed device blocks, reused across streams once idle; builds
    # and frees alternating between two streams must give identical forests
    import torch
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=12, count=60)
    dev = torch.from_numpy(P).cuda()
    base_i, base_c = ragged.Forest(dev, off).knn(6)
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    keep = []
    for i in range(6):
        s = streams[i % 2]
        with torch.cuda.stream(s):
            f = ragged.Forest(dev, off)
            idx, cnt = f.knn(6)
        s.synchronize()
        assert torch.equal(idx, base_i) and torch.equal(cnt, base_c), i
        keep.append(f)
        if len(keep) > 1:
            keep.pop(0)  # frees the forest built on the other stream


def test_capture_needs_device_forest(gpu):
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=5, count=12)
    with pytest.raises(ValueError):
        ragged.Forest(P, off).capture_knn(4)


def test_autotuned_settings_give_identical_results(gpu):
    import torch
    from pptk_b200 import _native as N
    from pptk_b200 import autotune, ragged
    P, off, _ = small_batch(seed=6, count=30)
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    ref_i, ref_c = f.knn(8)
    ref_n = f.normals(8)
    try:
        res = autotune.tune(lambda: f.knn(8), f.set_bucket, buckets=(16, 64), lane_spans=(-1, 0), repeats=1)
        assert res["bucket"] in (16, 64) and res["lane_span"] in (-1, 0) and len(res["table"]) == 4
        assert res["warm_bound"] in (0, 1) and res["topk_min"] in (0, 32) and res["warm_mult"] in (2, 3)
        assert len(res["knob_table"]) == 6
        for b, ls, wb, tk, wm in ((16, -1, 1, 0, 2), (64, 0, 0, 32, 3), (64, 256, 1, 16, 4), (32, 1024, 1, 8, 1),
                                  (res["bucket"], res["lane_span"], res["warm_bound"], res["topk_min"],
                                   res["warm_mult"])):
            f.set_bucket(b)
            N.tune_set("lane_span", ls)
            N.tune_set("warm_bound", wb)
            N.tune_set("topk_min", tk)
            N.tune_set("warm_mult", wm)
            i, c = f.knn(8)
            assert torch.equal(i, ref_i) and torch.equal(c, ref_c), (b, ls, wb, tk, wm)
            n = f.normals(8)
            assert torch.equal(torch.nan_to_num(n, nan=-9.0), torch.nan_to_num(ref_n, nan=-9.0)), (b, ls, wb, tk, wm)
    finally:
        N.tune_set("lane_span", 1024)
        N.tune_set("warm_bound", 1)
        N.tune_set("topk_min", 0)
        N.tune_set("warm_mult", 2)


def _same_forest(f, g):
    """Two forests over the same rows hold the same trees and answer alike."""
    import torch
    assert np.array_equal(f.valid_offsets, g.valid_offsets)
    assert np.array_equal(f.reverse_indices(), g.reverse_indices())
    for c in range(f.ncloud):
        assert np.array_equal(f.ref_nodes(c), g.ref_nodes(c)), c
    fi, fc = f.knn(8)
    gi, gc = g.knn(8)
    assert torch.equal(fi, gi) and torch.equal(fc, gc)
    fn, gn = f.normals(8), g.normals(8)
    assert torch.equal(torch.nan_to_num(fn, nan=-9.0), torch.nan_to_num(gn, nan=-9.0))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rebuild_equals_a_fresh_forest(gpu, dtype):
    # capture mode: the trees rebuilt in place from new coordinates of the
    # same rows (dropped rows moved, clouds squeezed and stretched) are the
    # trees a new forest builds
    import torch
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=21, count=30, dtype=dtype)
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    f.capture_ready()
    rng = np.random.default_rng(3)
    for trial in range(3):
        Q = P * rng.uniform(0.5, 2.0, size=(1, 3)).astype(dtype) + rng.normal(size=P.shape).astype(dtype) * 0.01
        Q[rng.integers(0, len(Q), 50)] = np.nan
        if trial == 2:
            Q = P.copy()
        dq = torch.from_numpy(Q).cuda()
        f.rebuild(dq)
        _same_forest(f, ragged.Forest(dq, off))


def test_captured_build_and_queries_replay(gpu):
    # one graph: rebuild from a fixed input tensor, kNN, normals; each
    # replay after a refill equals a new forest over the refilled points
    import torch
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=22, count=25)
    buf = torch.from_numpy(P).cuda()
    f = ragged.Forest(buf, off)
    cap, out = f.capture_pipeline(buf, 8)
    rng = np.random.default_rng(4)
    for trial in range(3):
        Q = P + rng.normal(size=P.shape).astype(np.float32) * 0.05
        Q[rng.integers(0, len(Q), 20)] = np.nan
        buf.copy_(torch.from_numpy(Q))
        for t in out.values():
            t.fill_(-7)
        cap.replay()
        torch.cuda.synchronize()
        cap.check()
        g = ragged.Forest(torch.from_numpy(Q).cuda(), off)
        gi, gc = g.knn(8)
        assert torch.equal(out["indices"], gi) and torch.equal(out["counts"], gc), trial
        assert torch.equal(torch.nan_to_num(out["normals"], nan=-9.0), torch.nan_to_num(g.normals(8), nan=-9.0))
        f.refresh()
        assert np.array_equal(f.valid_offsets, g.valid_offsets)


def _chain_cloud(n_clusters=60, per=400, seed=0):
    """Clusters at x = 2^-j: every widest-axis midpoint split peels off one
    cluster, so segments above the per-CTA subtree size last ~50 levels."""
    rng = np.random.default_rng(seed)
    parts = []
    for j in range(n_clusters):
        c = rng.normal(size=(per, 3)) * (1e-3 * 2.0 ** -j)
        c[:, 0] += 2.0 ** -j
        parts.append(c)
    return np.concatenate(parts).astype(np.float32)


def test_rebuild_deeper_than_planned_is_refused(gpu):
    import torch
    from pptk_b200 import ragged
    deep = _chain_cloud()
    n = len(deep)
    P = np.random.default_rng(1).random((n, 3), dtype=np.float32)
    off = np.array([0, n])
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    f.capture_ready()
    with pytest.raises(NotImplementedError, match="more tree levels"):
        f.rebuild(torch.from_numpy(deep).cuda())
    # the same points through a captured pipeline: the status word says so
    buf = torch.from_numpy(P).cuda()
    g = ragged.Forest(buf, off)
    cap, _ = g.capture_pipeline(buf, 8, normals=False)
    buf.copy_(torch.from_numpy(deep))
    cap.replay()
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match="deeper tree"):
        cap.check()
    # a new forest over those points is fine
    h = ragged.Forest(torch.from_numpy(deep).cuda(), off)
    assert h.n_valid == n


def test_rebuild_argument_checks(gpu):
    import torch
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=23, count=10)
    f = ragged.Forest(torch.from_numpy(P).cuda(), off)
    with pytest.raises(ValueError):
        f.rebuild(torch.from_numpy(P).cuda())  # not capture-ready
    f.capture_ready()
    with pytest.raises(ValueError):
        f.rebuild(torch.from_numpy(P[:-1]).cuda())
    with pytest.raises(ValueError):
        f.rebuild(torch.from_numpy(P.astype(np.float64)).cuda())
    with pytest.raises(TypeError):
        f.rebuild(P)
    with pytest.raises(ValueError):
        ragged.Forest(P, off).capture_ready()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fused_knn_normals_equal_the_separate_calls(gpu, dtype):
    # one walk per point answers the self kNN and the normal; with exact
    # duplicates the query point's place among the zero-distance points
    # follows the index rule (a cloud of 40 copies of one point, and a cloud
    # whose first 20 rows repeat one point)
    import torch
    from pptk_b200 import ragged
    P, off, clouds = small_batch(seed=31, count=20, dtype=dtype)
    rng = np.random.default_rng(5)
    dup = np.repeat(rng.random((1, 3)), 40, axis=0).astype(dtype)
    mixed = rng.random((300, 3)).astype(dtype)
    mixed[:20] = mixed[0]
    P = np.concatenate([P, dup, mixed])
    off = np.concatenate([off, [off[-1] + 40, off[-1] + 340]])
    for dev in (False, True):
        f = ragged.Forest(torch.from_numpy(P).cuda() if dev else P, off)
        for k in (4, 16, 24):
            i2, c2, n2 = f.knn_normals(k)
            i1, c1 = f.knn(k)
            n1 = f.normals(k)
            if dev:
                i1, c1, n1, i2, c2, n2 = (x.cpu().numpy() for x in (i1, c1, n1, i2, c2, n2))
            assert np.array_equal(i1, i2) and np.array_equal(c1, c2), (dev, k)
            assert np.array_equal(np.nan_to_num(n1, nan=-9.0), np.nan_to_num(n2, nan=-9.0)), (dev, k)


def test_fused_pipeline_replay_equals_separate_calls(gpu):
    import torch
    from pptk_b200 import ragged
    P, off, _ = small_batch(seed=32, count=25)
    buf = torch.from_numpy(P).cuda()
    f = ragged.Forest(buf, off)
    cap, out = f.capture_pipeline(buf, 16)
    Q = P + np.random.default_rng(8).normal(size=P.shape).astype(np.float32) * 0.02
    buf.copy_(torch.from_numpy(Q))
    cap.replay()
    torch.cuda.synchronize()
    cap.check()
    g = ragged.Forest(torch.from_numpy(Q).cuda(), off)
    gi, gc = g.knn(16)
    assert torch.equal(out["indices"], gi) and torch.equal(out["counts"], gc)
    assert torch.equal(torch.nan_to_num(out["normals"], nan=-9.0), torch.nan_to_num(g.normals(16), nan=-9.0))
