"""Drop-in for ``pptk.kdtree``: ``_build`` and ``_query`` on the GPU.

Mirrors ``pptk/kdtree/kdtree_wrapper.cpp`` (``Build`` :281-304, ``Query``
:340-412): the same arguments, defaults, query forms, result layout and
exception types.  Points and queries may be numpy arrays (results come back
as numpy) or CUDA torch tensors (results stay on the device).

Two additional entry points return whole result arrays instead of a Python
list of per-query arrays: ``knn`` (dense m x k, -1 padded) and ``rnear``
(CSR offsets + indices).
"""
import ctypes
import math

import numpy as np

from . import _native as N
from ._args import as_points_2d, cast_as_float_rounded, extract_indices

_UNSET = object()
_FLOAT_CODES = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}


class KdTree:
    """Handle of a device-resident k-d tree (what ``_build`` returns in place
    of the reference's PyCapsule).  The tree keeps its own copy of the
    points; the memory is released when the handle is garbage collected."""

    __slots__ = ("_h", "n", "n_valid", "dim", "dtype", "device", "__weakref__")

    def __init__(self, handle, device):
        self._h = handle
        n, nv, dim, dt, nrec, depth = (ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int(), ctypes.c_int(),
                                       ctypes.c_int64(), ctypes.c_int())
        N.call("pptkg_tree_info", handle, ctypes.byref(n), ctypes.byref(nv), ctypes.byref(dim), ctypes.byref(dt),
               ctypes.byref(nrec), ctypes.byref(depth))
        self.n, self.n_valid, self.dim = n.value, nv.value, dim.value
        self.dtype = N.CODE_DTYPES[dt.value]
        self.device = device

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().pptkg_tree_free(h)
            except Exception:
                pass
            self._h = None

    def save(self, path):
        """Writes the device tree to `path` (pptkg_tree_save); kdtree.load
        puts it back on a device without rebuilding."""
        _save_handle(self._h, path)

    def num_points(self):
        """Number of stored (valid) points, the reference's num_points()."""
        return self.n_valid

    def reverse_indices(self):
        """Tree position -> original row (numpy int32)."""
        out = np.empty(self.n_valid, np.int32)
        N.call("pptkg_tree_reverse_indices", self._h, N.ptr(out), N.MEM_HOST, None)
        return out

    def ref_nodes(self):
        """The reference node list (preorder, 5 columns: split dim, split
        index, split value, has left child, has right child)."""
        cnt = ctypes.c_int64()
        N.call("pptkg_tree_ref_nodes", self._h, None, 0, ctypes.byref(cnt))
        out = np.empty((cnt.value, 5), np.float64)
        N.call("pptkg_tree_ref_nodes", self._h, N.ptr(out), cnt.value, ctypes.byref(cnt))
        return out

    def set_bucket(self, bucket):
        """Re-cuts the traversal hierarchy at `bucket` points per leaf."""
        N.call("pptkg_tree_set_bucket", self._h, int(bucket), self._stream())

    def _stream(self):
        if self.device is None:
            return None
        return N.torch_stream(self.device)


def _build(data, numprocs=-1, maxleafsize=10, emptysplit=0.2):
    """Builds a k-d tree.

    Parameters
    ----------
    data : n x k numpy array (or CUDA torch tensor) of float32, float64 or an
        integer type (int8 ... uint64), k in [2, 4].  Integer trees are
        built in their own type and answer queries in float32, the
        reference's distance type for integers.
    numprocs : int, optional
        Accepted for compatibility; the build runs on the GPU.
    maxleafsize : int, optional
        Leaf nodes have at most this many points. Default: 10.
    emptysplit : float, optional
        Empty splits are performed for gap ratios greater than this value. Default: 0.2

    Returns
    -------
    tree : KdTree handle, meant to be passed into ``_query``.
    """
    try:
        numprocs = int(numprocs)
        maxleafsize = int(maxleafsize)
        emptysplit = float(emptysplit)
    except (TypeError, ValueError) as e:
        raise TypeError("Build(): failed parsing arguments") from e
    a, m, dim = as_points_2d(data, "Build()")
    if dim not in (2, 3, 4):
        raise RuntimeError(f"PerformAction(): Invalid k-d tree dim = {dim}.")
    if N.is_torch_cuda(a):
        import torch
        tcodes = {torch.float32: 0, torch.float64: 1, torch.int8: 2, torch.int16: 3, torch.int32: 4,
                  torch.int64: 5, torch.uint8: 6}
        if a.dtype not in tcodes:
            raise RuntimeError(f"PerformAction_(): Invalid k-d tree type_num (dtype {a.dtype}).")
        a = a.contiguous()
        code = tcodes[a.dtype]
        mem, stream, device = N.MEM_DEVICE, N.torch_stream(a.device), a.device
    else:
        if a.dtype not in N.DTYPE_CODES:
            raise RuntimeError(f"PerformAction_(): Invalid k-d tree type_num (dtype {a.dtype}).")
        a = np.ascontiguousarray(a)
        code = N.DTYPE_CODES[a.dtype]
        mem, stream, device = N.MEM_HOST, None, None
    h = ctypes.c_void_p()
    N.call("pptkg_tree_build", N.ptr(a), int(m), int(dim), code, mem, maxleafsize, emptysplit, stream,
           ctypes.byref(h), where="Build()")
    return KdTree(h, device)


def _parse_k_dmax(k, dmax):
    # Query(): k and dmax conventions (kdtree_wrapper.cpp:354-390)
    if k is _UNSET:
        kk = 1
    elif k is None:
        kk = -1
    else:
        kk = int(k)
        if kk <= 0:
            raise ValueError(f"Query(): encountered negative k={kk}")
    if dmax is _UNSET or dmax is None:
        dm = math.inf
    else:
        dm = cast_as_float_rounded(dmax)
        if dm < 0.0:
            raise ValueError(f"Query(): encountered negative dmax {dm:f}")
    return kk, dm


def _check_tree(kdtree):
    if not isinstance(kdtree, KdTree) or not kdtree._h:
        raise TypeError("Query(): first arg must be capsule of a KdTreeStruct pointer")


class _Batch:
    """One resolved query batch: point rows or stored-row indices."""

    def __init__(self, tree, queries):
        self.points = None
        self.indices = None
        self.qdtype = 0
        self.torch = False
        self.mem = N.MEM_HOST
        self.stream = tree._stream()
        if queries is None:
            # indices 0 .. num_points()-1 (kdtree_wrapper.cpp:176-179)
            self.m = tree.n_valid
            return
        if isinstance(queries, slice):
            raise NotImplementedError("QueryTreeAction::Perform(): slice-based query not yet implemented")
        if N.is_torch_cuda(queries):
            import torch
            self.torch = True
            self.mem = N.MEM_DEVICE
            self.stream = N.torch_stream(queries.device)
            if queries.dim() == 2:
                if queries.shape[1] != tree.dim:
                    raise ValueError(f"QueryTreeAction::Perform(): query point dim = {queries.shape[1]} "
                                     f"(expecting dim = {tree.dim}).")
                q = queries
                if q.dtype not in (torch.float32, torch.float64):
                    q = q.to(torch.float32 if tree.dtype.kind in "iu" else torch.float64)
                self.points = q.contiguous()
                self.qdtype = 0 if q.dtype == torch.float32 else 1
                self.m = int(q.shape[0])
                return
            idx = extract_indices(queries.cpu().numpy(), tree.n_valid)
            self.indices = torch.from_numpy(idx).to(queries.device)
            self.m = int(idx.shape[0])
            return
        if isinstance(queries, np.ndarray) and queries.ndim == 2:
            if queries.shape[1] != tree.dim:
                raise ValueError(f"QueryTreeAction::Perform(): query point dim = {queries.shape[1]} "
                                 f"(expecting dim = {tree.dim}).")
            q = queries
            if q.dtype not in _FLOAT_CODES:
                # integer trees compute in float32 (one conversion per
                # coordinate, as the reference's (DistT)q); float trees
                # take other query types through float64
                q = q.astype(np.float32 if tree.dtype.kind in "iu" else np.float64)
            self.points = np.ascontiguousarray(q)
            self.qdtype = _FLOAT_CODES[self.points.dtype]
            self.m = self.points.shape[0]
            return
        idx = extract_indices(queries, tree.n_valid)
        if idx is None:
            raise TypeError(f"QueryTreeAction::Perform(): could not use object of type "
                            f"{type(queries).__name__} as query input.")
        self.indices = idx
        self.m = idx.shape[0]

    def new(self, shape, dtype):
        if self.torch:
            import torch
            tdt = {np.int32: torch.int32, np.int64: torch.int64}[dtype]
            dev = (self.points if self.points is not None else self.indices).device
            return torch.empty(shape, dtype=tdt, device=dev)
        return np.empty(shape, dtype)


def knn(kdtree, queries=None, k=1, dmax=math.inf):
    """Dense kNN: (indices m x k int32, -1 padded; counts m int32), in
    ascending distance.  Point queries use KNearestNeighbors, index queries
    (or None) KNearestNeighborsSelf."""
    _check_tree(kdtree)
    k = int(k)
    if k <= 0:
        raise ValueError(f"Query(): encountered negative k={k}")
    dmax = cast_as_float_rounded(dmax)
    b = _Batch(kdtree, queries)
    idx = b.new((b.m, k), np.int32)
    cnt = b.new((b.m,), np.int32)
    if b.points is not None:
        N.call("pptkg_knn", kdtree._h, N.ptr(b.points), b.m, b.qdtype, b.mem, k, dmax, N.ptr(idx), N.ptr(cnt),
               b.stream, where="Query()")
    else:
        N.call("pptkg_knn_self", kdtree._h, N.ptr(b.indices), b.m, b.mem, k, dmax, N.ptr(idx), N.ptr(cnt),
               b.stream, where="Query()")
    return idx, cnt


def rnear(kdtree, queries=None, dmax=0.0):
    """r-near in CSR form: (offsets m+1 int64, indices int32); the hits of
    query i are indices[offsets[i]:offsets[i+1]] in the reference's order."""
    _check_tree(kdtree)
    dmax = cast_as_float_rounded(dmax)
    b = _Batch(kdtree, queries)
    return _rnear(kdtree, b, dmax)


def _rnear(kdtree, b, dmax):
    off = b.new((b.m + 1,), np.int64)
    total = ctypes.c_int64()
    N.call("pptkg_rnear_count", kdtree._h, N.ptr(b.points), N.ptr(b.indices), b.m, b.qdtype, b.mem, dmax,
           N.ptr(off), ctypes.byref(total), b.stream, where="Query()")
    out = b.new((max(total.value, 0),), np.int32)
    N.call("pptkg_rnear_fill", kdtree._h, N.ptr(b.points), N.ptr(b.indices), b.m, b.qdtype, b.mem, dmax,
           N.ptr(off), N.ptr(out), b.stream, where="Query()")
    return off, out


def _rows_from_dense(idx, cnt, k):
    if b_all_full(cnt, k):
        return list(idx)
    c = cnt.tolist() if isinstance(cnt, np.ndarray) else cnt.cpu().tolist()
    return [idx[i, :c[i]] for i in range(len(c))]


def b_all_full(cnt, k):
    if isinstance(cnt, np.ndarray):
        return bool((cnt == k).all())
    return bool((cnt == k).all().item())


def _query(kdtree, queries, k=_UNSET, dmax=_UNSET, numprocs=-1):
    """Query k-d tree for nearest neighbors.

    Query points can be specified by one of the following ways
    (n is the number of points in the k-d tree and m the number of queries):

        1. k-d points (m x k numpy array)
        2. integer indices (list or numpy array of m integers; negative integers supported)
        3. boolean selection mask on the n points used to build the k-d tree (numpy array of n bools)

    For each query point, returns up to k nearest neighbors that have
    distances strictly less than dmax from the query point (k=None: all
    points within dmax).

    Returns
    -------
    results: list of m numpy arrays of integer indices
    """
    kk, dm = _parse_k_dmax(k, dmax)
    _check_tree(kdtree)
    b = _Batch(kdtree, queries)
    form = "QueryWithPoints()" if b.points is not None else "QueryWithIndices()"
    if kk > 0:
        idx = b.new((b.m, kk), np.int32)
        cnt = b.new((b.m,), np.int32)
        if b.points is not None:
            N.call("pptkg_knn", kdtree._h, N.ptr(b.points), b.m, b.qdtype, b.mem, kk, dm, N.ptr(idx), N.ptr(cnt),
                   b.stream, where=form)
        else:
            N.call("pptkg_knn_self", kdtree._h, N.ptr(b.indices), b.m, b.mem, kk, dm, N.ptr(idx), N.ptr(cnt),
                   b.stream, where=form)
        return _rows_from_dense(idx, cnt, kk)
    if dm != math.inf:
        off, out = _rnear(kdtree, b, dm)
        o = off.tolist() if isinstance(off, np.ndarray) else off.cpu().tolist()
        return [out[o[i]:o[i + 1]] for i in range(b.m)]
    raise ValueError(f"{form}: k = {kk} and dmax = {dm:f} is an invalid combination.")


def _save_handle(h, path):
    size = ctypes.c_int64()
    N.call("pptkg_tree_save", h, None, 0, ctypes.byref(size), where="save()")
    buf = np.empty(size.value, np.uint8)
    N.call("pptkg_tree_save", h, N.ptr(buf), size.value, ctypes.byref(size), where="save()")
    with open(path, "wb") as f:
        f.write(buf.tobytes())


def _load_handle(path, device=None):
    data = np.fromfile(path, dtype=np.uint8)
    h = ctypes.c_void_p()
    if device is not None:
        import torch
        with torch.cuda.device(device):
            N.call("pptkg_tree_load", N.ptr(data), data.size, None, ctypes.byref(h), where="load()")
    else:
        N.call("pptkg_tree_load", N.ptr(data), data.size, None, ctypes.byref(h), where="load()")
    return h


def load(path, device=None):
    """A KdTree read back from a file written by KdTree.save, on `device`
    (a CUDA device index or torch.device; default: the current device).
    Damaged files raise ValueError."""
    return KdTree(_load_handle(path, device), device)
