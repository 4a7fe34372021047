"""Points with a cached device tree (the callers of _query) and the
neighbourhood PCA route, against direct queries and a float64 numpy
evaluation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_points_nbhds_follow_the_buffer(gpu):
    from pptk_b200.points import Points, points
    rng = np.random.default_rng(0)
    X = rng.random((20_000, 3)).astype(np.float32)
    P = points(X)
    t = gpu.kdtree._build(X)
    q = [0, 5, 19_999]
    assert all(np.array_equal(a, b) for a, b in zip(P.nbhds(q, k=8), gpu.kdtree._query(t, q, k=8)))
    assert P._update_kd_tree() is None  # cached: no rebuild
    # moving a point next to point 5 changes point 5's neighbourhood
    P[7] = X[5] + np.float32(1e-6)
    assert P._update_kd_tree() is not None  # the write forces a rebuild
    got = P.nbhds([5], k=2)[0]
    assert 7 in got.tolist()
    X2 = X.copy()
    X2[7] = X[5] + np.float32(1e-6)
    t2 = gpu.kdtree._build(X2)
    assert np.array_equal(got, gpu.kdtree._query(t2, [5], k=2)[0])
    # r-near form and the lazy expression
    r = P.nbhds(P[:10].view(np.ndarray), k=None, r=0.02)
    r2 = gpu.kdtree._query(t2, X2[:10], k=None, dmax=0.02)
    assert all(np.array_equal(a, b) for a, b in zip(r, r2))
    lazy = P.NBHDS(k=4)
    assert len(lazy) == len(P)
    ev = lazy.evaluate(chunk=7000)
    ref = gpu.kdtree._query(t2, None, k=4)
    assert len(ev) == len(ref) and all(np.array_equal(a, b) for a, b in zip(ev, ref))
    di, dc = P.nbhds_dense(k=4)
    assert np.array_equal(di, np.stack(ref))


def test_nbhd_pca_matches_float64(gpu):
    from pptk_b200 import pca
    from pptk_b200.points import Points, points
    rng = np.random.default_rng(1)
    X = rng.random((30_000, 3)).astype(np.float32)
    X[:, 2] *= 0.05
    P = points(X)
    nb = P.nbhds(np.arange(0, 30_000, 3), k=12)
    w, V = pca.nbhd_pca(X, nb)
    Y = np.stack([X[i].astype(np.float64) for i in nb])  # m x 12 x 3
    Y = Y - Y.mean(1, keepdims=True)
    C = np.einsum("mki,mkj->mij", Y, Y) / Y.shape[1]
    w64, V64 = np.linalg.eigh(C)
    assert np.allclose(w, w64, rtol=1e-4, atol=1e-7 * np.abs(w64).max())
    gap = (w64[:, 1] - w64[:, 0]) / w64[:, 2]
    ok = gap > 1e-3
    dots = np.abs((V[:, :, 0].astype(np.float64) * V64[:, :, 0]).sum(1))
    assert (dots[ok] > 1 - 1e-5).all()
    # the dense kNN form and the CSR form give the same matrices
    di, dc = P.nbhds_dense(np.arange(0, 30_000, 3), k=12)
    C1 = pca.nbhd_covariance(X, (di, dc))
    off = np.arange(0, 12 * len(nb) + 1, 12, dtype=np.int64)
    C2 = pca.nbhd_covariance(X, (off, np.concatenate(nb).astype(np.int32)))
    assert np.array_equal(C1, C2)
    with pytest.raises(RuntimeError):
        pca.nbhd_covariance(X, [np.array([0, 30_000])])


def test_eigh_list_matches_lapack(gpu):
    # vfuncs._eigh's calling form: a list of float32 3 x 3 arrays in, a list
    # of (w, V) pairs out with V[:, j] the j-th eigenvector; only the lower
    # triangle is read
    from pptk_b200 import pca
    rng = np.random.default_rng(2)
    X = []
    for i in range(500):
        Y = rng.normal(size=(3, 3))
        A = (Y @ Y.T).astype(np.float32)
        if i % 5 == 0:
            A = np.asfortranarray(A)  # any memory layout
        if i % 7 == 0:
            A[0, 2] += np.float32(5.0)  # the upper triangle is ignored
        X.append(A)
    out = pca.eigh_list(X)
    assert isinstance(out, list) and len(out) == len(X)
    for A, (w, V) in zip(X, out):
        assert w.dtype == np.float32 and V.dtype == np.float32 and w.shape == (3,) and V.shape == (3, 3)
        S = np.tril(A).astype(np.float64)
        S = S + np.tril(S, -1).T
        wl, Vl = np.linalg.eigh(S)
        assert np.allclose(w, wl, rtol=1e-5, atol=1e-5 * np.abs(wl).max())
        gap = np.diff(wl) / max(np.abs(wl).max(), 1e-30)
        for j in range(3):
            if (j == 0 or gap[j - 1] > 1e-3) and (j == 2 or gap[j] > 1e-3):
                assert abs(float(V[:, j].astype(np.float64) @ Vl[:, j])) > 1 - 1e-5
