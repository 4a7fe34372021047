"""GPU parity of estimate_normals and the batched 3x3 eigensolve.

Known answers follow the reference's tests/test_estimate_normals.py; the
general check is against the FP64 oracle (float64 covariance of the oracle's
neighbourhoods + LAPACK eigh): normals agree to |dot| >= 1 - 1e-6 and
eigenvalues to 1e-5 of the largest eigenvalue, except neighbourhoods whose
two smallest eigenvalues nearly coincide (relative gap < 1e-4), where the
normal direction is not defined by the data; those are counted.
"""
import os

import numpy as np
import pytest

from _util import angle_error

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DOT_TOL = 1e-6
EVAL_TOL = 1e-5
GAP_EXCLUDE = 1e-4


def collinear():
    y = np.zeros((10, 3), dtype=np.float64)
    y[:, 0] = np.arange(10)
    return y


EVALS = np.array([2.0 / 3] + [5.0 / 4] * 8 + [2.0 / 3])
EVECS = np.array([[1.0, 0.0, 0.0]] * 10)
SIZES = np.array([3] + [4] * 8 + [3])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_output_types_known_answer(gpu, dtype):
    en = gpu.estimate_normals
    y = collinear().astype(dtype)
    for ev_, all_, nb_ in [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]:
        z = en(y, 4, 3, output_eigenvalues=ev_, output_all_eigenvectors=all_, output_neighborhood_sizes=nb_,
               verbose=False)
        vshape = (10, 3, 3) if all_ else (10, 3)
        if not ev_ and not nb_:
            assert isinstance(z, np.ndarray) and z.shape == vshape
            continue
        assert isinstance(z, tuple) and len(z) == 3
        assert z[0].shape == vshape and z[0].dtype == dtype
        assert (z[1] is None) == (not ev_) and (z[2] is None) == (not nb_)
        if ev_:
            assert z[1].shape == ((10, 3) if all_ else (10,))
            if all_:
                assert np.allclose(z[1][:, -1], EVALS)
        if nb_:
            assert z[2].dtype == np.int32 and np.array_equal(z[2], SIZES)
        if all_:
            assert np.allclose(z[0][:, -1, :], EVECS)


def test_subsample_known_answer(gpu):
    en = gpu.estimate_normals
    y = collinear()
    s = [0, 3, 4, -1]
    mask = np.zeros(10, dtype=bool)
    mask[s] = True
    for sub in (mask, s):
        z = en(y, 4, 3, subsample=sub, output_eigenvalues=True, output_all_eigenvectors=True,
               output_neighborhood_sizes=True, verbose=False)
        sel = [0, 3, 4, 9]
        assert np.allclose(z[0][:, -1, :], EVECS[sel])
        assert np.allclose(z[1][:, -1], EVALS[sel])
        assert np.array_equal(z[2], SIZES[sel])
    with pytest.raises(ValueError):
        en(y, 4, 3, subsample=np.zeros(2, dtype=bool), verbose=False)


def test_argument_errors(gpu):
    en = gpu.estimate_normals
    y = collinear()
    with pytest.raises(ValueError):
        en(y, 4, 0.0, verbose=False)
    with pytest.raises(ValueError):
        en(y, 0, 1.0, verbose=False)
    with pytest.raises(ValueError):
        en(y, -1, np.inf, verbose=False)
    with pytest.raises(TypeError):
        en(y.astype(np.int32), 4, 1.0, verbose=False)
    with pytest.raises(RuntimeError):
        en(y, "a", 1.0, verbose=False)


def _check_against_fp64(port, P, k, r, gpu_out, label):
    ev, ew, sz = gpu_out
    _, _, osz, nb = port.port_estimate_normals(P, k, r, num_eigen=3, want_nbrs=True)
    assert np.array_equal(sz, osz), label
    w, V, _ = port.normals_fp64(P, nb)
    gap = (w[:, 1] - w[:, 0]) / np.maximum(np.abs(w[:, 2]), 1e-300)
    ok = gap >= GAP_EXCLUDE
    dots = np.abs((ev[:, 0, :].astype(np.float64) * V[:, 0, :]).sum(1))
    assert (dots[ok] >= 1 - DOT_TOL).all(), (label, np.sort(dots[ok])[:5])
    scale = np.abs(w[:, 2:3])
    assert (np.abs(ew.astype(np.float64) - w) <= EVAL_TOL * scale + 1e-30).all(), label
    return int((~ok).sum()), angle_error(ev[:, 0, :], V[:, 0, :])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_normals_match_fp64_oracle(gpu, port, dtype):
    # config-1 shape: 200k uniform points, k = 16, r = inf
    P = np.random.default_rng(0).random((200_000, 3)).astype(dtype)
    out = gpu.estimate_normals(P, 16, np.inf, output_eigenvalues=True, output_all_eigenvectors=True,
                               output_neighborhood_sizes=True, verbose=False)
    excluded, ang = _check_against_fp64(port, P, 16, np.inf, out, str(dtype))
    assert excluded < len(P) * 1e-3
    assert np.percentile(ang, 99) <= 1e-4


@pytest.mark.parametrize("dtype,precision", [(np.float64, "auto"), (np.float32, "fp64"), (np.float32, "auto")])
def test_eigenvalues_relative_to_each_eigenvalue(gpu, port, dtype, precision):
    # eigenvalues against the FP64 oracle, each to 1e-5 of itself (a floor
    # of 1e-12 of the largest for eigenvalues at zero).  The FP32 path
    # (float32 input, precision "auto") meets that for the two larger
    # eigenvalues; its smallest keeps the absolute bound of 1e-5 of the
    # largest: an FP32 eigensolve resolves an eigenvalue only to a few
    # float32 ulps of the largest, which is more than 1e-5 of the smallest
    # once the two differ by more than ~1e2 (a planar neighbourhood)
    P = np.random.default_rng(2).random((100_000, 3)).astype(dtype)
    ev, ew, sz = gpu.estimate_normals(P, 16, np.inf, output_eigenvalues=True, output_all_eigenvectors=True,
                                      output_neighborhood_sizes=True, verbose=False, precision=precision)
    _, _, osz, nb = port.port_estimate_normals(P, 16, np.inf, num_eigen=3, want_nbrs=True)
    assert np.array_equal(sz, osz)
    w, _, _ = port.normals_fp64(P, nb)
    lmax = np.abs(w[:, 2:3])
    err = np.abs(ew.astype(np.float64) - w)
    rel_ok = err <= EVAL_TOL * np.abs(w) + 1e-12 * lmax
    if dtype == np.float32 and precision == "auto":
        assert rel_ok[:, 1:].all(), np.max(err[:, 1:] / np.abs(w[:, 1:]))
        assert (err[:, 0] <= EVAL_TOL * lmax[:, 0]).all()
    else:
        assert rel_ok.all(), np.max(err / (np.abs(w) + 1e-300))


def test_normals_with_radius_and_rnear_neighbourhoods(gpu, port):
    P = np.random.default_rng(1).random((40_000, 3)).astype(np.float32)
    out = gpu.estimate_normals(P, 20, 0.05, output_eigenvalues=True, output_all_eigenvectors=True,
                               output_neighborhood_sizes=True, verbose=False)
    _, _, osz, _ = port.port_estimate_normals(P, 20, 0.05, num_eigen=3, want_nbrs=True)
    assert np.array_equal(out[2], osz)
    # r-near neighbourhoods (k = -1)
    ev, ew, sz = gpu.estimate_normals(P, -1, 0.03, output_eigenvalues=True, output_all_eigenvectors=True,
                                      output_neighborhood_sizes=True, verbose=False)
    pev, pew, psz = port.port_estimate_normals(P, -1, 0.03, num_eigen=3)
    assert np.array_equal(sz, psz)
    ok = sz >= 5
    gap = (pew[:, 1] - pew[:, 0]) / np.maximum(pew[:, 2], 1e-30)
    ok &= gap > 1e-3
    assert (angle_error(ev[ok, 0], pev[ok, 0]) < 2e-3).all()


def test_rnear_normals_warp_per_query_matches_packets(gpu):
    # r-near neighbourhoods (k = -1) of small batches run one warp per query
    # (rnear_warp_queries); sizes must match the packet walk exactly and the
    # FP64-solved normals and eigenvalues to rounding, for all points and a
    # subsample
    from pptk_b200 import _native as N
    P = np.random.default_rng(6).random((30_000, 3)).astype(np.float32)
    sub = np.arange(0, len(P), 7, dtype=np.int64)
    default = N.tune_get("rnear_warp_queries")
    out = {}
    try:
        for wq in (0, 1 << 30):
            N.tune_set("rnear_warp_queries", wq)
            out[wq] = (gpu.estimate_normals(P, -1, 0.04, output_eigenvalues=True, output_all_eigenvectors=True,
                                            output_neighborhood_sizes=True, verbose=False),
                       gpu.estimate_normals(P, -1, 0.04, subsample=sub, output_eigenvalues=True,
                                            output_all_eigenvectors=True, output_neighborhood_sizes=True,
                                            verbose=False))
    finally:
        N.tune_set("rnear_warp_queries", default)
    (ev0, ew0, sz0), (sv0, sw0, ss0) = out[0]
    (ev1, ew1, sz1), (sv1, sw1, ss1) = out[1 << 30]
    assert np.array_equal(sz0, sz1) and np.array_equal(ss0, ss1)
    ok = sz0 >= 5
    ok &= (ew0[:, 1] - ew0[:, 0]) / np.maximum(ew0[:, 2], 1e-30) > 1e-3
    assert (angle_error(ev0[ok, 0], ev1[ok, 0]) < 1e-5).all()
    np.testing.assert_allclose(ew0[ok], ew1[ok], rtol=1e-5, atol=1e-9)
    oks = ss0 >= 5
    oks &= (sw0[:, 1] - sw0[:, 0]) / np.maximum(sw0[:, 2], 1e-30) > 1e-3
    assert (angle_error(sv0[oks, 0], sv1[oks, 0]) < 1e-5).all()
    # rows with NaN coordinates: size 0 and NaN results in both forms
    P2 = P[:3000].copy()
    P2[::97] = np.nan
    res = []
    try:
        for wq in (0, 1 << 30):
            N.tune_set("rnear_warp_queries", wq)
            res.append(gpu.estimate_normals(P2, -1, 0.05, output_neighborhood_sizes=True, verbose=False))
    finally:
        N.tune_set("rnear_warp_queries", default)
    (n0, _, z0), (n1, _, z1) = res
    assert np.array_equal(z0, z1) and (z0[::97] == 0).all()
    assert np.array_equal(np.isnan(n0), np.isnan(n1)) and np.isnan(n0[::97]).all()


def test_precision_split_on_offset_planes(gpu):
    # config-3 shape, reduced: thin patches 1e5 m from the origin, float64
    from pptk_b200 import synth
    P, true_n = synth.planar_patches(300_000, seed=3)
    n32 = gpu.estimate_normals(P, 24, np.inf, precision="fp32", verbose=False)
    n64 = gpu.estimate_normals(P, 24, np.inf, precision="fp64", verbose=False)
    inl = np.isfinite(true_n[:, 0])
    a = angle_error(n32[inl], n64[inl])
    assert np.percentile(a, 99) <= 1e-4


def test_torch_inputs(gpu):
    import torch
    P = torch.rand(30_000, 3, device="cuda", dtype=torch.float64)
    z = gpu.estimate_normals(P, 10, np.inf, output_neighborhood_sizes=True, verbose=False)
    assert z[0].is_cuda and z[0].shape == (30_000, 3) and z[2].is_cuda
    zz = gpu.estimate_normals(P.cpu().numpy(), 10, np.inf, verbose=False)
    assert np.allclose(np.abs(z[0].cpu().numpy()), np.abs(zz))


def test_eigh3_batched(gpu):
    rng = np.random.default_rng(7)
    X = rng.normal(size=(10_000, 3, 3))
    A = X @ np.transpose(X, (0, 2, 1))
    for dt, tol in ((np.float64, 1e-10), (np.float32, 2e-5)):
        w, V = gpu.eigh3(A.astype(dt))
        wl, Vl = np.linalg.eigh(A)
        assert np.allclose(w, wl, rtol=tol, atol=tol * np.abs(wl).max(1, keepdims=True))
        gap = np.diff(wl, axis=1).min(1) / np.abs(wl).max(1)
        ok = gap > 1e-3
        assert (np.abs((V * Vl).sum(1))[ok] > 1 - 100 * tol).all()
        w2, V2 = gpu.eigh3(A.astype(dt), layout="rows")
        assert np.array_equal(V2, np.transpose(V, (0, 2, 1)))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_large_k_normals_match_fp64_oracle(gpu, port, dtype):
    # k above the register lists (64): device-memory heaps, FP64 covariance
    P = np.random.default_rng(7).random((30_000, 3)).astype(dtype)
    P[:, 2] *= 0.1
    for k, r in ((100, np.inf), (150, 0.08)):
        out = gpu.estimate_normals(P, k, r, output_eigenvalues=True, output_all_eigenvectors=True,
                                   output_neighborhood_sizes=True, verbose=False)
        excluded, ang = _check_against_fp64(port, P, k, r, out, f"{dtype} k={k}")
        assert excluded < len(P) * 1e-3
