"""Ragged batches: thousands of independent clouds built and queried together.

A ``Forest`` holds one k-d tree per cloud of a CSR batch (points concatenated,
``offsets[c]:offsets[c+1]`` the rows of cloud c).  Each tree is exactly the
tree ``pptk.kdtree._build`` gives for that cloud alone, but all clouds are
built in one device build pass and queried in one launch: warps are assigned
to clouds, each cloud's queries padded to whole warps, and every warp walks
its own cloud's tree.
"""
import ctypes
import math

import numpy as np

from . import _native as N

_CODES = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}


class Forest:
    """Device-resident trees of a ragged batch of clouds."""

    def __init__(self, points, offsets, maxleafsize=10, emptysplit=0.2):
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
        if off.ndim != 1 or off.size < 2:
            raise ValueError("offsets must hold at least two entries")
        if N.is_torch_cuda(points):
            import torch
            if points.dtype not in (torch.float32, torch.float64):
                raise TypeError("points must be float32 or float64")
            p = points.contiguous()
            code = 0 if p.dtype == torch.float32 else 1
            mem, self._stream, self.device = N.MEM_DEVICE, N.torch_stream(p.device), p.device
        else:
            p = np.ascontiguousarray(points)
            if p.dtype not in _CODES:
                raise TypeError("points must be float32 or float64")
            code = _CODES[p.dtype]
            mem, self._stream, self.device = N.MEM_HOST, None, None
        if p.ndim != 2 or p.shape[1] not in (2, 3, 4):
            raise ValueError("points must be (n, 2..4)")
        if off[0] != 0 or off[-1] != p.shape[0] or (np.diff(off) < 0).any():
            raise ValueError("offsets must start at 0, end at n and not decrease")
        self.n, self.dim = int(p.shape[0]), int(p.shape[1])
        self.dtype = np.dtype(np.float32) if code == 0 else np.dtype(np.float64)
        self.offsets = off
        self.ncloud = off.size - 1
        self._h = ctypes.c_void_p()
        N.call("pptkg_forest_build", N.ptr(p), self.n, self.dim, code, mem, N.ptr(off), self.ncloud, int(maxleafsize),
               float(emptysplit), self._stream, ctypes.byref(self._h), where="Forest()")
        vo = np.empty(self.ncloud + 1, np.int64)
        nc = ctypes.c_int()
        N.call("pptkg_forest_info", self._h, ctypes.byref(nc), N.ptr(vo))
        self.valid_offsets = vo
        self.n_valid = int(vo[-1])
        self._torch = mem == N.MEM_DEVICE

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().pptkg_tree_free(h)
            except Exception:
                pass
            self._h = None

    def _new(self, shape, dtype):
        if self._torch:
            import torch
            tdt = {np.dtype(np.int32): torch.int32, np.dtype(np.float32): torch.float32,
                   np.dtype(np.float64): torch.float64}[np.dtype(dtype)]
            return torch.empty(shape, dtype=tdt, device=self.device)
        return np.empty(shape, dtype)

    @property
    def _mem(self):
        return N.MEM_DEVICE if self._torch else N.MEM_HOST

    def reverse_indices(self):
        """Global tree position -> global input row."""
        out = np.empty(self.n_valid, np.int32)
        N.call("pptkg_tree_reverse_indices", self._h, N.ptr(out), N.MEM_HOST, None)
        return out

    def ref_nodes(self, cloud):
        """Reference node list of one cloud's tree (preorder, 5 columns)."""
        cnt = ctypes.c_int64()
        N.call("pptkg_forest_ref_nodes", self._h, int(cloud), None, 0, ctypes.byref(cnt))
        out = np.empty((cnt.value, 5), np.float64)
        N.call("pptkg_forest_ref_nodes", self._h, int(cloud), N.ptr(out), cnt.value, ctypes.byref(cnt))
        return out

    def save(self, path):
        """Writes the forest to `path`; Forest.load reads it back."""
        from .kdtree import _save_handle
        _save_handle(self._h, path)

    @classmethod
    def load(cls, path, offsets, device=None, torch_results=None):
        """A forest read back from Forest.save.  `offsets` are the clouds'
        input offsets (checked against the stored ones).  Results come back
        as CUDA tensors when torch_results (default: device given)."""
        from .kdtree import _load_handle
        self = cls.__new__(cls)
        self._h = _load_handle(path, device)
        nc = ctypes.c_int()
        N.call("pptkg_forest_info", self._h, ctypes.byref(nc), None)
        vo = np.empty(nc.value + 1, np.int64)
        N.call("pptkg_forest_info", self._h, ctypes.byref(nc), N.ptr(vo))
        off = np.asarray(offsets, dtype=np.int64)
        if off.size != nc.value + 1:
            raise ValueError("offsets do not match the stored forest")
        n = ctypes.c_int64()
        nv = ctypes.c_int64()
        dim = ctypes.c_int()
        dt = ctypes.c_int()
        nrec = ctypes.c_int64()
        depth = ctypes.c_int()
        N.call("pptkg_tree_info", self._h, ctypes.byref(n), ctypes.byref(nv), ctypes.byref(dim), ctypes.byref(dt),
               ctypes.byref(nrec), ctypes.byref(depth))
        if off[-1] != n.value:
            raise ValueError("offsets do not match the stored forest")
        self.n, self.dim = n.value, dim.value
        self.dtype = N.CODE_DTYPES[dt.value]
        self.offsets = off
        self.ncloud = nc.value
        self.valid_offsets = vo
        self.n_valid = int(vo[-1])
        self._torch = (device is not None) if torch_results is None else bool(torch_results)
        if self._torch:
            import torch
            self.device = torch.device("cuda", device if isinstance(device, int) else
                                       (torch.cuda.current_device() if device is None else torch.device(device).index))
            self._stream = N.torch_stream(self.device)
        else:
            self.device, self._stream = None, None
        return self

    def set_bucket(self, bucket):
        N.call("pptkg_tree_set_bucket", self._h, int(bucket), self._stream)

    def knn(self, k, dmax=math.inf, exclude_self=True):
        """k nearest neighbours of every point within its own cloud:
        (indices n x k as global rows, -1 padded; counts n)."""
        idx = self._new((self.n, int(k)), np.int32)
        cnt = self._new((self.n,), np.int32)
        N.call("pptkg_forest_knn", self._h, int(k), float(np.float32(dmax)), int(bool(exclude_self)), self._mem,
               N.ptr(idx), N.ptr(cnt), self._stream, where="Forest.knn()")
        return idx, cnt

    def normals(self, k, r=math.inf, output_eigenvalues=False, output_all_eigenvectors=False,
                output_neighborhood_sizes=False, precision="auto"):
        """estimate_normals over every cloud at once (same layouts)."""
        from .estimate_normals import PRECISIONS
        if self.dim != 3:
            raise TypeError("normals need 3-d points")
        ne = 3 if output_all_eigenvectors else 1
        ev = self._new((self.n, 3) if ne == 1 else (self.n, 3, 3), self.dtype)
        ew = self._new((self.n,) if ne == 1 else (self.n, 3), self.dtype) if output_eigenvalues else None
        sz = self._new((self.n,), np.int32) if output_neighborhood_sizes else None
        N.call("pptkg_forest_normals", self._h, int(k), ctypes.c_float(float(np.float32(r))), ne,
               PRECISIONS[precision], self._mem, N.ptr(ev), N.ptr(ew), N.ptr(sz), self._stream,
               where="Forest.normals()")
        if ew is None and sz is None:
            return ev
        return ev, ew, sz

    def knn_normals(self, k, r=math.inf, precision="auto"):
        """(indices, counts, normals): Forest.knn(k, dmax=r, exclude_self=True)
        and Forest.normals(k, r) from one traversal per point; each result
        equals the separate call."""
        from .estimate_normals import PRECISIONS
        if self.dim != 3:
            raise TypeError("normals need 3-d points")
        idx = self._new((self.n, int(k)), np.int32)
        cnt = self._new((self.n,), np.int32)
        ev = self._new((self.n, 3), self.dtype)
        N.call("pptkg_forest_knn_normals", self._h, int(k), ctypes.c_float(float(np.float32(r))), 1,
               PRECISIONS[precision], self._mem, N.ptr(idx), N.ptr(cnt), N.ptr(ev), None, None, self._stream,
               where="Forest.knn_normals()")
        return idx, cnt, ev

    # ------------------------------------------------------- rebuilds --
    def capture_ready(self):
        """Sizes the forest's device arrays for rebuilds from any coordinates
        of the same rows (capture mode).  After it, rebuild() and the
        pipeline of capture_pipeline() rebuild the trees in place, without
        host synchronisation."""
        if not self._torch:
            raise ValueError("capture mode needs a forest built from CUDA tensors")
        N.call("pptkg_forest_capture_ready", self._h, self._stream, where="Forest.capture_ready()")
        self._capture_mode = True

    def _check_points(self, points):
        import torch
        if not N.is_torch_cuda(points) or points.device != self.device:
            raise TypeError("points must be a CUDA tensor on the forest's device")
        want = torch.float32 if self.dtype == np.float32 else torch.float64
        if points.dtype != want or tuple(points.shape) != (self.n, self.dim) or not points.is_contiguous():
            raise ValueError(f"points must be a contiguous ({self.n}, {self.dim}) tensor of {self.dtype}")

    def refresh(self):
        """Reads the valid offsets of the last (re)build back (after captured
        rebuilds; waits for the device)."""
        vo = np.empty(self.ncloud + 1, np.int64)
        nc = ctypes.c_int()
        N.call("pptkg_forest_info", self._h, ctypes.byref(nc), N.ptr(vo))
        self.valid_offsets = vo
        self.n_valid = int(vo[-1])

    def rebuild(self, points):
        """Rebuilds every cloud's tree from new coordinates of the same rows
        (a contiguous CUDA tensor shaped like the build's points); the trees
        equal those Forest(points, offsets) builds.  Needs capture_ready()."""
        if not getattr(self, "_capture_mode", False):
            raise ValueError("rebuild needs capture_ready() first")
        self._check_points(points)
        N.call("pptkg_forest_rebuild", self._h, N.ptr(points), self._stream, where="Forest.rebuild()")
        self.refresh()

    def capture_pipeline(self, points, k, r=math.inf, knn=True, normals=True, dmax=math.inf, exclude_self=True,
                         precision="auto", fused=True):
        """(CapturedQuery, outputs): one CUDA graph that rebuilds the forest
        from `points` (a fixed CUDA tensor the caller refills between
        replays), then runs Forest.knn (k, dmax, exclude_self) and / or
        Forest.normals (k, r) into fixed tensors -- as one Forest.knn_normals
        traversal when both are asked for with exclude_self and dmax == r
        (unless fused=False).  outputs: {"indices", "counts", "normals"} as
        requested.  Calls capture_ready() if needed.  A replay whose points
        need a deeper tree than the first build's + 8 levels makes check()
        raise (build a new forest then)."""
        from .estimate_normals import PRECISIONS
        if not getattr(self, "_capture_mode", False):
            self.capture_ready()
        self._check_points(points)
        if normals and self.dim != 3:
            raise TypeError("normals need 3-d points")
        out = {}
        if knn:
            out["indices"] = self._new((self.n, int(k)), np.int32)
            out["counts"] = self._new((self.n,), np.int32)
        if normals:
            out["normals"] = self._new((self.n, 3), self.dtype)

        one_walk = (fused and knn and normals and exclude_self
                    and float(np.float32(dmax)) == float(np.float32(r)))

        def issue(stream):
            N.call("pptkg_forest_rebuild", self._h, N.ptr(points), stream, where="Forest.capture_pipeline()")
            if one_walk:
                N.call("pptkg_forest_knn_normals", self._h, int(k), ctypes.c_float(float(np.float32(r))), 1,
                       PRECISIONS[precision], self._mem, N.ptr(out["indices"]), N.ptr(out["counts"]),
                       N.ptr(out["normals"]), None, None, stream, where="Forest.capture_pipeline()")
                return
            if knn:
                N.call("pptkg_forest_knn", self._h, int(k), float(np.float32(dmax)), int(bool(exclude_self)),
                       self._mem, N.ptr(out["indices"]), N.ptr(out["counts"]), stream,
                       where="Forest.capture_pipeline()")
            if normals:
                N.call("pptkg_forest_normals", self._h, int(k), ctypes.c_float(float(np.float32(r))), 1,
                       PRECISIONS[precision], self._mem, N.ptr(out["normals"]), None, None, stream,
                       where="Forest.capture_pipeline()")

        return self._capture(issue), out

    # ------------------------------------------------------ graph capture --
    def _capture(self, issue):
        """Captures issue(stream) -- native forest calls into fixed output
        tensors -- into a CUDA graph.  The calls run once uncaptured first
        (they set up the forest's slot tables and load the kernels)."""
        import torch
        if not self._torch:
            raise ValueError("graph capture needs a forest built from CUDA tensors")
        sink = torch.zeros(1, dtype=torch.int32, device=self.device)
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            issue(N.torch_stream(self.device))
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            N.call("pptkg_set_status_sink", N.ptr(sink))
            try:
                issue(N.torch_stream(self.device))
            finally:
                N.call("pptkg_set_status_sink", None)
        return CapturedQuery(g, sink)

    def capture_knn(self, k, dmax=math.inf, exclude_self=True):
        """(CapturedQuery, (indices, counts)): Forest.knn captured into a CUDA
        graph; every replay() rewrites the two tensors."""
        idx = self._new((self.n, int(k)), np.int32)
        cnt = self._new((self.n,), np.int32)

        def issue(stream):
            N.call("pptkg_forest_knn", self._h, int(k), float(np.float32(dmax)), int(bool(exclude_self)), self._mem,
                   N.ptr(idx), N.ptr(cnt), stream, where="Forest.capture_knn()")

        return self._capture(issue), (idx, cnt)

    def capture_normals(self, k, r=math.inf, precision="auto"):
        """(CapturedQuery, normals): Forest.normals captured into a CUDA
        graph."""
        from .estimate_normals import PRECISIONS
        if self.dim != 3:
            raise TypeError("normals need 3-d points")
        ev = self._new((self.n, 3), self.dtype)

        def issue(stream):
            N.call("pptkg_forest_normals", self._h, int(k), ctypes.c_float(float(np.float32(r))), 1,
                   PRECISIONS[precision], self._mem, N.ptr(ev), None, None, stream, where="Forest.capture_normals()")

        return self._capture(issue), ev


class CapturedQuery:
    """A forest query captured into a CUDA graph.  replay() launches it on
    the current stream; check() waits for it and raises if a kernel check
    failed in any replay since the last check."""

    def __init__(self, graph, sink):
        self.graph = graph
        self.sink = sink

    def replay(self):
        self.graph.replay()

    def check(self):
        code = int(self.sink.item())
        if code:
            self.sink.zero_()
            if code in (20, 21):
                raise RuntimeError("captured forest rebuild: the points need a deeper tree than planned "
                                   f"(code {code}; build the forest again)")
            raise RuntimeError(f"captured forest query: device check failed (code {code})")
