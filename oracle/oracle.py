"""Test infrastructure: Python access to the oracle libraries.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, as the checker.  The product (``pptk_b200``) never
imports it.

* ``Port`` wraps ``oracle/libpptk_port.so``, the CPU restatement of the
  reference's k-d tree and normal estimation (``oracle/port.cpp``).
* ``Ref`` wraps ``oracle/_ref/libpptk_ref.so``, the reference's own k-d tree
  headers compiled in place (``oracle/ref_harness.cpp``); absent where the
  reference tree is not available and the library was not shipped along.
* ``normals_fp64`` is the FP64 normal oracle: float64 covariance of each
  neighbourhood (estimate_normals.cpp:84-88) and LAPACK ``numpy.linalg.eigh``.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libpptk_port.so")
REF_SO = os.path.join(HERE, "_ref", "libpptk_ref.so")

DTYPES = {
    np.dtype(np.float32): 0, np.dtype(np.float64): 1,
    np.dtype(np.int8): 2, np.dtype(np.int16): 3, np.dtype(np.int32): 4, np.dtype(np.int64): 5,
    np.dtype(np.uint8): 6, np.dtype(np.uint16): 7, np.dtype(np.uint32): 8, np.dtype(np.uint64): 9,
}

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_dbl = ctypes.c_double
_flt = ctypes.c_float


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _bind(lib, prefix):
    sig = {
        "build": (_vp, [_vp, _i64, _i32, _i32, _i32, _dbl]),
        "free": (None, [_vp]),
        "num_valid": (_i64, [_vp]),
        "reverse_indices": (None, [_vp, _vp]),
        "tree_nodes": (_i64, [_vp, _vp]),
        "knn_self": (None, [_vp, _vp, _i64, _i32, _dbl, _vp, _vp, _i32]),
        "rnear": (None, [_vp, _vp, _i64, _i32, _dbl, _vp, _vp, _i32]),
        "rnear_self": (None, [_vp, _vp, _i64, _dbl, _vp, _vp, _i32]),
    }
    if prefix == "port":
        sig["knn"] = (None, [_vp, _vp, _i64, _i32, _i32, _dbl, _vp, _vp, _vp, _vp, _i32])
        sig["tree_points"] = (None, [_vp, _vp])
        sig["estimate_normals"] = (None, [_vp, _i64, _i32, _i32, _flt, _vp, _i64, _i32, _vp, _vp, _vp, _vp,
                                          _i32])
        sig["eigh3"] = (None, [_vp, _i64, _i32, _vp, _vp])
    else:
        sig["knn"] = (None, [_vp, _vp, _i64, _i32, _i32, _dbl, _vp, _vp, _i32])
        sig["estimate_normals"] = (None, [_vp, _i64, _i32, _i32, _flt, _vp, _i64, _i32, _vp, _vp, _vp, _i32,
                                          _vp])
        sig["tree_normals"] = (None, [_vp, _vp, _vp, _i64, _i32, _flt, _i32, _vp, _vp, _vp, _i32])
    sig["max_threads"] = (_i32, [])
    for name, (res, args) in sig.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.restype = res
        fn.argtypes = args
    return lib


class _Tree:
    """A k-d tree built by one of the oracle libraries."""

    def __init__(self, lib, prefix, points, maxleafsize=10, emptysplit=0.2):
        pts = np.ascontiguousarray(points)
        if pts.ndim != 2 or pts.dtype not in DTYPES:
            raise TypeError("oracle tree needs an (n, dim) array of a supported dtype")
        self._lib, self._p = lib, prefix
        self.points = pts
        self.n, self.dim = pts.shape
        self.dtype = pts.dtype
        self._h = self._fn("build")(_ptr(pts), self.n, self.dim, DTYPES[pts.dtype], int(maxleafsize),
                                    float(emptysplit))
        if not self._h:
            raise ValueError("oracle build failed (dtype/dim)")

    def _fn(self, name):
        return getattr(self._lib, f"{self._p}_{name}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._fn("free")(h)
            self._h = None

    @property
    def num_valid(self):
        return int(self._fn("num_valid")(self._h))

    def reverse_indices(self):
        out = np.empty(self.num_valid, np.int32)
        self._fn("reverse_indices")(self._h, _ptr(out))
        return out

    def nodes(self):
        cnt = self._fn("tree_nodes")(self._h, None)
        out = np.empty((cnt, 5), np.float64)
        self._fn("tree_nodes")(self._h, _ptr(out))
        return out

    def _queries(self, q):
        q = np.ascontiguousarray(q)
        if q.dtype not in (self.dtype, np.dtype(np.float32), np.dtype(np.float64)):
            q = q.astype(np.float64)
        return q

    def knn_self(self, qidx, k, dmax=np.inf, nthreads=0):
        qidx = np.ascontiguousarray(qidx, dtype=np.int32)
        m = len(qidx)
        idx = np.empty((m, k), np.int32)
        cnt = np.empty(m, np.int32)
        self._fn("knn_self")(self._h, _ptr(qidx), m, k, float(dmax), _ptr(idx), _ptr(cnt), nthreads)
        return idx, cnt

    def rnear(self, q, dmax, nthreads=0):
        q = self._queries(q)
        m = q.shape[0]
        off = np.empty(m + 1, np.int64)
        self._fn("rnear")(self._h, _ptr(q), m, DTYPES[q.dtype], float(dmax), _ptr(off), None, nthreads)
        out = np.empty(int(off[-1]), np.int32)
        self._fn("rnear")(self._h, _ptr(q), m, DTYPES[q.dtype], float(dmax), _ptr(off), _ptr(out), nthreads)
        return off, out

    def rnear_self(self, qidx, dmax, nthreads=0):
        qidx = np.ascontiguousarray(qidx, dtype=np.int32)
        m = len(qidx)
        off = np.empty(m + 1, np.int64)
        self._fn("rnear_self")(self._h, _ptr(qidx), m, float(dmax), _ptr(off), None, nthreads)
        out = np.empty(int(off[-1]), np.int32)
        self._fn("rnear_self")(self._h, _ptr(qidx), m, float(dmax), _ptr(off), _ptr(out), nthreads)
        return off, out


class PortTree(_Tree):
    def __init__(self, points, maxleafsize=10, emptysplit=0.2):
        super().__init__(port_lib(), "port", points, maxleafsize, emptysplit)

    def tree_points(self):
        out = np.empty((self.num_valid, self.dim), np.float64)
        self._fn("tree_points")(self._h, _ptr(out))
        return out

    def knn(self, q, k, dmax=np.inf, nthreads=0, with_pos=False):
        """(idx m x k, cnt m[, pos m x k, d2 m x k]) in (dist2, point index) order."""
        q = self._queries(q)
        m = q.shape[0]
        idx = np.empty((m, k), np.int32)
        cnt = np.empty(m, np.int32)
        pos = np.empty((m, k), np.int32) if with_pos else None
        d2 = np.empty((m, k), np.float64) if with_pos else None
        self._fn("knn")(self._h, _ptr(q), m, DTYPES[q.dtype], k, float(dmax), _ptr(idx), _ptr(cnt), _ptr(pos),
                        _ptr(d2), nthreads)
        return (idx, cnt, pos, d2) if with_pos else (idx, cnt)


class RefTree(_Tree):
    def __init__(self, points, maxleafsize=10, emptysplit=0.2):
        super().__init__(ref_lib(), "ref", points, maxleafsize, emptysplit)

    def knn(self, q, k, dmax=np.inf, nthreads=0):
        q = self._queries(q)
        m = q.shape[0]
        idx = np.empty((m, k), np.int32)
        cnt = np.empty(m, np.int32)
        self._fn("knn")(self._h, _ptr(q), m, DTYPES[q.dtype], k, float(dmax), _ptr(idx), _ptr(cnt), nthreads)
        return idx, cnt

    def normals(self, rows, k, r=np.inf, nthreads=0):
        """The restated normal loop over this (resident) tree for the given
        rows of its input: (normals m x 3, sizes m)."""
        if self.dim != 3 or self.dtype not in (np.float32, np.float64):
            raise TypeError("normals need a 3-d float32/float64 tree")
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        m = len(rows)
        ev = np.empty((m, 3), self.dtype)
        sz = np.empty(m, np.int32)
        self._fn("tree_normals")(self._h, _ptr(self.points), _ptr(rows), m, int(k), float(r), 1, _ptr(ev), None,
                                 _ptr(sz), nthreads)
        return ev, sz


_port = None
_ref = None


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            from . import build_oracle  # noqa: F401  (package-relative when imported as oracle.oracle)
            build_oracle.build_port()
        _port = _bind(ctypes.CDLL(PORT_SO), "port")
    return _port


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError("reference harness not built (oracle/_ref/libpptk_ref.so)")
        _ref = _bind(ctypes.CDLL(REF_SO), "ref")
    return _ref


def _normals_call(lib, prefix, points, k, r, subsample=None, num_eigen=1, nthreads=0, want_nbrs=False):
    pts = np.ascontiguousarray(points)
    if pts.dtype not in (np.float32, np.float64) or pts.ndim != 2 or pts.shape[1] != 3:
        raise TypeError("points must be (n, 3) float32/float64")
    n = pts.shape[0]
    sub = None if subsample is None else np.ascontiguousarray(subsample, dtype=np.int32)
    m = n if sub is None else len(sub)
    shape_v = (m, 3) if num_eigen == 1 else (m, 3, 3)
    shape_w = (m,) if num_eigen == 1 else (m, 3)
    ev = np.empty(shape_v, pts.dtype)
    ew = np.empty(shape_w, pts.dtype)
    sz = np.empty(m, np.int32)
    fn = getattr(lib, f"{prefix}_estimate_normals")
    if prefix == "port":
        nb = np.empty((m, k), np.int32) if (want_nbrs and k > 0) else None
        fn(_ptr(pts), n, DTYPES[pts.dtype], int(k), float(r), _ptr(sub), m, num_eigen, _ptr(ev), _ptr(ew),
           _ptr(sz), _ptr(nb), nthreads)
        return (ev, ew, sz, nb) if want_nbrs else (ev, ew, sz)
    bt = ctypes.c_double(0.0)
    fn(_ptr(pts), n, DTYPES[pts.dtype], int(k), float(r), _ptr(sub), m, num_eigen, _ptr(ev), _ptr(ew), _ptr(sz),
       nthreads, ctypes.byref(bt))
    return ev, ew, sz, bt.value


def port_estimate_normals(points, k, r, subsample=None, num_eigen=1, nthreads=0, want_nbrs=False):
    """Restated estimate_normals: (evecs, evals, sizes[, neighbourhoods])."""
    return _normals_call(port_lib(), "port", points, k, r, subsample, num_eigen, nthreads, want_nbrs)


def ref_estimate_normals(points, k, r, subsample=None, num_eigen=1, nthreads=0):
    """estimate_normals over the reference tree: (evecs, evals, sizes, build seconds)."""
    return _normals_call(ref_lib(), "ref", points, k, r, subsample, num_eigen, nthreads)


def port_eigh3(A):
    A = np.ascontiguousarray(A)
    m = A.shape[0]
    w = np.empty((m, 3), A.dtype)
    V = np.empty((m, 3, 3), A.dtype)
    port_lib().port_eigh3(_ptr(A), m, DTYPES[A.dtype], _ptr(w), _ptr(V))
    return w, V


def normals_fp64(points, nbr_idx, counts=None):
    """FP64 oracle: eigenvalues (m, 3) ascending and eigenvectors (m, 3, 3)
    with [i, j, :] the j-th eigenvector, from float64 covariances of the
    neighbourhoods nbr_idx (m x k, -1 padded)."""
    P = np.asarray(points, dtype=np.float64)
    nb = np.asarray(nbr_idx)
    valid = nb >= 0
    cnt = valid.sum(1) if counts is None else np.asarray(counts)
    X = P[np.where(valid, nb, 0)]
    X = np.where(valid[..., None], X, 0.0)
    mean = X.sum(1) / np.maximum(cnt, 1)[:, None]
    Xc = np.where(valid[..., None], X - mean[:, None, :], 0.0)
    C = np.einsum("mki,mkj->mij", Xc, Xc) / np.maximum(cnt, 1)[:, None, None]
    w, V = np.linalg.eigh(C)
    return w, np.transpose(V, (0, 2, 1)), C
