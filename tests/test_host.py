"""Host-side logic and the C ABI boundary (CPU only: no compute calls)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "pptkg.h")).read()
    return re.findall(r"PPTKG_API\s+\w+\s+(pptkg_\w+)\s*\(", src)


def test_library_loads_and_exports_every_declared_symbol():
    from pptk_b200 import _native
    lib = _native.lib()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert lib.pptkg_version() >= 100
    # every binding the Python layer declares exists in the header
    assert set(_native.SIGNATURES) <= set(syms)


def test_c_abi_rejects_bad_arguments_without_a_gpu():
    # argument checks run before any device call
    from pptk_b200 import _native as N
    lib = N.lib()
    h = ctypes.c_void_p()
    assert lib.pptkg_tree_build(None, 10, 3, 0, N.MEM_HOST, 10, 0.2, None, ctypes.byref(h)) == N.E_INVALID
    assert lib.pptkg_tree_build(None, 0, 7, 0, N.MEM_HOST, 10, 0.2, None, ctypes.byref(h)) == N.E_TYPE
    assert lib.pptkg_tree_build(None, 0, 3, 11, N.MEM_HOST, 10, 0.2, None, ctypes.byref(h)) == N.E_TYPE
    assert lib.pptkg_knn(None, None, 0, 0, 0, 1, 1.0, None, None, None) == N.E_INVALID
    code, msg = N.last_error()
    assert code == N.E_INVALID and "null tree" in msg
    with pytest.raises(ValueError):
        N.check(N.E_INVALID, "x")


def test_tuning_knobs_validate_and_round_trip():
    # process-wide traversal knobs: defaults, accepted ranges, rejected values
    from pptk_b200 import _native as N
    lib = N.lib()
    for name, default, good, bad in (("lane_span", 1024, (-1, 0, 64, 1 << 20), (-2,)),
                                     ("rnear_warp_queries", 262144, (0, 1, 1 << 30), (-1,)),
                                     ("warm_bound", 1, (0, 1), (-1, 2)),
                                     ("topk_min", 0, (4, 8, 16, 32, 64, 0), (-1, 3, 65, 128)),
                                     ("warm_mult", 2, (1, 3, 8, 2), (0, 9, -1))):
        assert N.tune_get(name) == default
        try:
            for v in good:
                N.tune_set(name, v)
                assert N.tune_get(name) == v
            for v in bad:
                assert lib.pptkg_tune_set(name.encode(), ctypes.c_int64(v)) == N.E_INVALID
                assert N.tune_get(name) == good[-1]
        finally:
            N.tune_set(name, default)
    assert lib.pptkg_tune_set(b"no_such_knob", ctypes.c_int64(1)) == N.E_INVALID


def test_index_extraction_follows_reference_rules():
    from pptk_b200._args import extract_indices
    assert extract_indices([0, -1, 3], 5).tolist() == [0, 4, 3]
    assert extract_indices(np.array([2, -5]), 5).tolist() == [2, 0]
    m = np.zeros(5, bool)
    m[[1, 3]] = True
    assert extract_indices(m, 5).tolist() == [1, 3]
    assert extract_indices(np.int64(4), 5).tolist() == [4]
    assert extract_indices("x", 5) is None
    with pytest.raises(ValueError):
        extract_indices(np.zeros(4, bool), 5)
    with pytest.raises(RuntimeError):
        extract_indices([5], 5)
    with pytest.raises(RuntimeError):
        extract_indices([-6], 5)
    with pytest.raises(ValueError):
        extract_indices(np.array([1.0, 2.0]), 5)
    with pytest.raises(TypeError):
        extract_indices([1, "a"], 5)


def test_k_and_dmax_conventions():
    from pptk_b200.kdtree import _UNSET, _parse_k_dmax
    assert _parse_k_dmax(_UNSET, _UNSET) == (1, math.inf)
    assert _parse_k_dmax(None, 0.5) == (-1, float(np.float32(0.5)))
    assert _parse_k_dmax(3, None) == (3, math.inf)
    assert _parse_k_dmax(2, 0.1)[1] == float(np.float32(0.1))  # rounded through float32
    for bad in ((0, _UNSET), (-2, _UNSET), (1, -0.5)):
        with pytest.raises(ValueError):
            _parse_k_dmax(*bad)
    with pytest.raises(ValueError):
        _parse_k_dmax("a", _UNSET)
    with pytest.raises(ValueError):
        _parse_k_dmax(1, "a")


def test_estimate_normals_argument_checks_precede_device_work():
    from pptk_b200 import estimate_normals
    y = np.zeros((10, 3))
    with pytest.raises(ValueError, match="r must be positive"):
        estimate_normals(y, 4, 0.0, verbose=False)
    with pytest.raises(ValueError, match="k cannot be zero"):
        estimate_normals(y, 0, 1.0, verbose=False)
    with pytest.raises(ValueError, match="invalid combo"):
        estimate_normals(y, -1, np.inf, verbose=False)
    with pytest.raises(RuntimeError, match="Failed to parse"):
        estimate_normals(y, 1.5, 1.0, verbose=False)
    with pytest.raises(TypeError):
        estimate_normals(y.astype(np.int32), 4, 1.0, verbose=False)
    with pytest.raises(TypeError):
        estimate_normals("points", 4, 1.0, verbose=False)


def test_build_argument_checks_precede_device_work():
    from pptk_b200 import kdtree
    with pytest.raises(RuntimeError, match="Invalid k-d tree dim"):
        kdtree._build(np.zeros((5, 5), np.float32))
    with pytest.raises(TypeError):
        kdtree._build("points")
    with pytest.raises(TypeError):
        kdtree._build(np.zeros((5, 3), np.float32), maxleafsize="x")
    with pytest.raises(RuntimeError, match="type_num"):
        kdtree._build(np.zeros((5, 3), np.complex64))


def test_synthetic_workloads_are_seeded():
    from pptk_b200 import synth
    a = synth.lidar_scene(20_000, seed=2)
    b = synth.lidar_scene(20_000, seed=2)
    assert a.dtype == np.float32 and a.shape == (20_000, 3) and np.array_equal(a, b)
    assert np.abs(a[:, :2]).max() < 110 and np.isfinite(a).all()
    p, n = synth.planar_patches(10_000, seed=3)
    assert p.dtype == np.float64 and (p[:, 0] > 9e4).all()
    s = synth.ragged_sizes(64)
    assert (s >= 1000).all() and (s <= 200_000).all()


def test_points_track_writes_through_views():
    import importlib
    PM = importlib.import_module("pptk_b200.points")
    from pptk_b200.points import Points, points
    P = points(np.zeros((10, 3), np.float32))
    assert not P.flags.writeable
    with pytest.raises(ValueError):
        np.ndarray.__setitem__(P, 0, 1.0)  # plain writes are refused
    g0 = P._gen.value
    v = P[2:5]
    assert v._gen is P._gen  # a view shares the buffer's write counter
    v += 1
    assert P._gen.value > g0 and P[2, 0] == 1.0 and not v.flags.writeable
    v[0, 1] = 7.0
    assert P[2, 1] == 7.0 and P._gen.value > g0 + 1
    c = P.copy()
    assert c._gen is not P._gen and not c.flags.writeable
    with pytest.raises(TypeError):
        np.zeros((4, 3)).view(Points)  # a plain array cannot report its writes
    assert len(P.NBHDS(queries=[1, 2, 3], k=2)) == 3
    # every in-place operator marks the buffer
    for op in ("__iadd__", "__isub__", "__imul__", "__itruediv__", "__ipow__"):
        g = P._gen.value
        getattr(P, op)(np.float32(1.0))
        assert P._gen.value == g + 1, op
    Q = points(np.arange(12, dtype=np.int32).reshape(4, 3))
    for op in ("__ifloordiv__", "__imod__", "__ilshift__", "__irshift__", "__iand__", "__ixor__", "__ior__"):
        g = Q._gen.value
        getattr(Q, op)(np.int32(1))
        assert Q._gen.value == g + 1, op
    # constructors
    assert (PM.zeros((2, 3)) == 0).all() and (PM.ones((2, 3)) == 1).all() and PM.empty((2, 3)).shape == (2, 3)
    assert (PM.ones_like(P) == 1).all() and PM.zeros_like(P).dtype == P.dtype and PM.rand(3, 3).shape == (3, 3)
    assert isinstance(PM.points(P, copy=False), Points) and PM.points(P, copy=False)._gen is P._gen


def test_eigh_list_argument_errors():
    # checked before any device work (vfuncs.cpp:1241-1270 contract)
    from pptk_b200 import pca
    with pytest.raises(TypeError):
        pca.eigh_list(np.eye(3, dtype=np.float32))
    with pytest.raises(ValueError):
        pca.eigh_list([])
    with pytest.raises(TypeError):
        pca.eigh_list([np.eye(3)])  # float64
    with pytest.raises(TypeError):
        pca.eigh_list([[1.0, 0.0]])
    with pytest.raises(ValueError):
        pca.eigh_list([np.zeros((2, 3), np.float32)])
    with pytest.raises(ValueError):
        pca.eigh_list([np.zeros((1, 3, 3), np.float32)])
    with pytest.raises(NotImplementedError):
        pca.eigh_list([np.eye(4, dtype=np.float32)])
