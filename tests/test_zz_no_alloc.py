"""The allocation-free normals entry point, through the C ABI (needs a B200).

pptkg_tree_normals_noalloc serves callers that cannot allocate device
memory -- code running under another framework that reserved the GPU's
memory up front, or latency-critical loops that cannot afford a cudaMalloc.
Its scratch is a static device array, shared by all calls, so these tests
check two calls in a row against the allocating entry point
(pptkg_tree_normals) with the tolerances of the other normal tests: every
top-k capacity class (k = 3, 8, 16), both precision modes, explicit rows and
the first-m-rows form, and a cloud whose neighbourhoods all go through the
FP64 re-solve queue that lives in the static array.  They also check the
size limits and that host pointers are refused.  The file name makes pytest
collect it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DOT_TOL = 1e-6
EVAL_TOL = 1e-5
MAX_QUERIES = 65536


def _lib():
    from pptk_b200 import _native as N
    lib = N.lib()
    fn = lib.pptkg_tree_normals_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return N, lib


def _need_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


_TREES = {}


def _uniform_tree(dtype):
    """One 120k-point tree per dtype, shared by the parametrized cases."""
    torch = _need_cuda()
    if dtype not in _TREES:
        from pptk_b200 import kdtree
        gen = torch.Generator(device="cuda").manual_seed(11)
        P = torch.rand((120_000, 3), device="cuda", dtype=getattr(torch, dtype), generator=gen)
        idx = torch.randperm(len(P), device="cuda", generator=gen)[:50_000].to(torch.int32)
        _TREES[dtype] = (P, kdtree._build(P), idx)
    return _TREES[dtype]


def _run_both(tree, idx, m, k, prec, tdt, calls=2):
    """(allocating results, [no-alloc results of `calls` calls in a row])."""
    torch = _need_cuda()
    N, lib = _lib()
    stream = N.torch_stream()
    iptr = N.ptr(idx) if idx is not None else None
    ev = torch.empty((m, 3, 3), device="cuda", dtype=tdt)
    ew = torch.empty((m, 3), device="cuda", dtype=tdt)
    sz = torch.empty((m,), device="cuda", dtype=torch.int32)
    # the allocating entry reads NULL indices as all rows, so the first m
    # rows are passed to it explicitly
    rows = idx if idx is not None else torch.arange(m, device="cuda", dtype=torch.int32)
    N.call("pptkg_tree_normals", tree._h, N.ptr(rows), m, N.MEM_DEVICE, k, ctypes.c_float(np.inf), 3, prec,
           N.ptr(ev), N.ptr(ew), N.ptr(sz), stream)
    ref = [x.cpu().numpy() for x in (ev, ew, sz)]
    got = []
    for _ in range(calls):
        ev = torch.full((m, 3, 3), float("nan"), device="cuda", dtype=tdt)
        ew = torch.full((m, 3), float("nan"), device="cuda", dtype=tdt)
        sz = torch.full((m,), -7, device="cuda", dtype=torch.int32)
        torch.cuda.synchronize()
        rc = lib.pptkg_tree_normals_noalloc(tree._h, iptr, m, k, ctypes.c_float(np.inf), 3, prec, N.ptr(ev),
                                            N.ptr(ew), N.ptr(sz), stream)
        assert rc == 0, N.last_error()
        got.append([x.cpu().numpy() for x in (ev, ew, sz)])
    return ref, got


def _assert_close(got, ref):
    assert np.array_equal(got[2], ref[2])
    dots = np.abs((got[0].astype(np.float64) * ref[0].astype(np.float64)).sum(-1))
    assert (dots >= 1 - DOT_TOL).all()
    scale = np.abs(ref[1][:, 2:3]).astype(np.float64)
    assert (np.abs(got[1].astype(np.float64) - ref[1]) <= EVAL_TOL * scale + 1e-30).all()


@pytest.mark.parametrize("rows", ["indices", "first_rows"])
@pytest.mark.parametrize("prec", ["auto", "fp64"])
@pytest.mark.parametrize("k", [3, 8, 16])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_noalloc_normals_match_allocating_entry(dtype, k, prec, rows):
    torch = _need_cuda()
    N, _ = _lib()
    P, tree, idx = _uniform_tree(dtype)
    m = len(idx) if rows == "indices" else 40_000
    p = N.PREC_AUTO if prec == "auto" else N.PREC_FP64
    ref, got = _run_both(tree, idx if rows == "indices" else None, m, k, p, getattr(torch, dtype))
    for g in got:  # two calls in a row share the same static scratch
        _assert_close(g, ref)


def _cross_clusters():
    """64 clusters, each a centre point with two points on each of three
    orthogonal axes (randomly rotated per cluster) at distances 1, 0.5 and
    0.5 (1 + 1e-4): every 7-point neighbourhood is one cluster, with a
    relative eigen-gap near 5e-5, below the 1e-3 threshold of the FP64
    re-solve."""
    rng = np.random.default_rng(16)
    c = np.stack(np.meshgrid(*[np.arange(4.0) * 5.0] * 3), -1).reshape(-1, 3)
    offs = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 0.5, 0], [0, -0.5, 0],
                     [0, 0, 0.5 * (1 + 1e-4)], [0, 0, -0.5 * (1 + 1e-4)]])
    R = np.linalg.qr(rng.normal(size=(len(c), 3, 3)))[0]
    return (c[:, None, :] + offs[None] @ np.transpose(R, (0, 2, 1))).reshape(-1, 3).astype(np.float32)


def test_noalloc_fp64_resolve_queue_in_static_scratch():
    # every neighbourhood is queued for the FP64 re-solve, whose queue is
    # part of the static array.  Both calls must equal the allocating entry
    # (whose queue is allocated) bit for bit, and their normals must be the
    # FP64 ones: an FP32 solve alone is off by about 1e-3 rad at this gap.
    torch = _need_cuda()
    N, _ = _lib()
    from pptk_b200 import kdtree
    from _util import angle_error
    P = torch.from_numpy(_cross_clusters()).cuda()
    tree = kdtree._build(P)
    m = len(P)
    ref, got = _run_both(tree, None, m, 7, N.PREC_AUTO, torch.float32)
    fp64, _ = _run_both(tree, None, m, 7, N.PREC_FP64, torch.float32, calls=0)
    w = fp64[1].astype(np.float64)
    assert ((w[:, 1] - w[:, 0]) / w[:, 2] < 1e-3).all()  # all neighbourhoods take the re-solve
    assert (ref[2] == 7).all()
    for g in got:
        _assert_close(g, ref)
        assert np.array_equal(g[0], ref[0]) and np.array_equal(g[1], ref[1])
        assert angle_error(g[0][:, 0, :], fp64[0][:, 0, :]).max() <= 1e-5


def test_noalloc_rejects_sizes_beyond_its_limit():
    torch = _need_cuda()
    N, lib = _lib()
    from pptk_b200 import kdtree
    P = torch.rand((MAX_QUERIES + 10, 3), device="cuda")
    tree = kdtree._build(P)
    out = torch.empty((MAX_QUERIES + 10, 3), device="cuda")
    stream = N.torch_stream(P.device)
    rc = lib.pptkg_tree_normals_noalloc(tree._h, None, MAX_QUERIES + 1, 8, ctypes.c_float(np.inf), 1, N.PREC_AUTO,
                                        N.ptr(out), None, None, stream)
    assert rc == N.E_INVALID and "65536" in N.last_error()[1]
    rc = lib.pptkg_tree_normals_noalloc(tree._h, None, 100, 17, ctypes.c_float(np.inf), 1, N.PREC_AUTO, N.ptr(out),
                                        None, None, stream)
    assert rc == N.E_INVALID
    # within the limit it works on the same tree
    rc = lib.pptkg_tree_normals_noalloc(tree._h, None, 1000, 8, ctypes.c_float(np.inf), 1, N.PREC_AUTO, N.ptr(out),
                                        None, None, stream)
    assert rc == 0 and torch.isfinite(out[:1000]).all()


def test_noalloc_refuses_host_pointers():
    # host memory given where device memory is required is an error before
    # any kernel reads it
    torch = _need_cuda()
    N, lib = _lib()
    from pptk_b200 import kdtree
    P = torch.rand((5000, 3), device="cuda")
    tree = kdtree._build(P)
    stream = N.torch_stream(P.device)
    dev_out = torch.empty((100, 3), device="cuda")
    host_idx = np.arange(100, dtype=np.int32)
    rc = lib.pptkg_tree_normals_noalloc(tree._h, N.ptr(host_idx), 100, 8, ctypes.c_float(np.inf), 1, N.PREC_AUTO,
                                        N.ptr(dev_out), None, None, stream)
    assert rc == N.E_INVALID and "device memory" in N.last_error()[1]
    host_out = np.empty((100, 3), np.float32)
    dev_idx = torch.arange(100, device="cuda", dtype=torch.int32)
    rc = lib.pptkg_tree_normals_noalloc(tree._h, N.ptr(dev_idx), 100, 8, ctypes.c_float(np.inf), 1, N.PREC_AUTO,
                                        N.ptr(host_out), None, None, stream)
    assert rc == N.E_INVALID and "device memory" in N.last_error()[1]
    rc = lib.pptkg_tree_normals_noalloc(tree._h, N.ptr(dev_idx), 100, 8, ctypes.c_float(np.inf), 1, N.PREC_AUTO,
                                        N.ptr(dev_out), None, None, stream)
    assert rc == 0 and torch.isfinite(dev_out).all()
