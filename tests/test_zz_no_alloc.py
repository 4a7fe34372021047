"""The allocation-free normals entry point, through the C ABI (needs a B200).

pptkg_tree_normals_noalloc serves callers that cannot allocate device
memory -- code running under another framework that reserved the GPU's
memory up front, or latency-critical loops that cannot afford a cudaMalloc.
Its scratch is a static device array, shared by all calls, so this test
checks two calls in a row against the allocating entry point
(pptkg_tree_normals) with the tolerances of the other normal tests, plus the
size limit.  The file name makes pytest collect it last.
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


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_noalloc_normals_match_allocating_entry(dtype):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    N, lib = _lib()
    from pptk_b200 import kdtree
    tdt = getattr(torch, dtype)
    gen = torch.Generator(device="cuda").manual_seed(11)
    P = torch.rand((120_000, 3), device="cuda", dtype=tdt, generator=gen)
    tree = kdtree._build(P)
    m, k = 50_000, 16
    idx = torch.randperm(len(P), device="cuda", generator=gen)[:m].to(torch.int32)
    stream = N.torch_stream(P.device)

    def allocating():
        ev = torch.empty((m, 3, 3), device="cuda", dtype=tdt)
        ew = torch.empty((m, 3), device="cuda", dtype=tdt)
        sz = torch.empty((m,), device="cuda", dtype=torch.int32)
        N.call("pptkg_tree_normals", tree._h, N.ptr(idx), m, N.MEM_DEVICE, k, ctypes.c_float(np.inf), 3,
               N.PREC_AUTO, N.ptr(ev), N.ptr(ew), N.ptr(sz), stream)
        return ev, ew, sz

    def no_alloc():
        ev = torch.full((m, 3, 3), float("nan"), device="cuda", dtype=tdt)
        ew = torch.full((m, 3), float("nan"), device="cuda", dtype=tdt)
        sz = torch.full((m,), -7, device="cuda", dtype=torch.int32)
        torch.cuda.synchronize()
        rc = lib.pptkg_tree_normals_noalloc(tree._h, N.ptr(idx), m, k, ctypes.c_float(np.inf), 3, N.PREC_AUTO,
                                            N.ptr(ev), N.ptr(ew), N.ptr(sz), stream)
        assert rc == 0, N.last_error()
        return ev, ew, sz

    ref = [x.cpu().numpy() for x in allocating()]
    for _ in range(2):  # two calls in a row share the same static scratch
        got = [x.cpu().numpy() for x in no_alloc()]
        assert np.array_equal(got[2], ref[2])
        dots = np.abs((got[0].astype(np.float64) * ref[0].astype(np.float64)).sum(-1))
        assert (dots >= 1 - DOT_TOL).all()
        scale = np.abs(ref[1][:, 2:3]).astype(np.float64)
        assert (np.abs(got[1].astype(np.float64) - ref[1]) <= EVAL_TOL * scale + 1e-30).all()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
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
