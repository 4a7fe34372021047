"""Points with a cached device k-d tree: the hot-path callers of pptk's
``_query`` (pptk/points/points.py:140-166, expr.py:397-424).

``Points`` is an ndarray subclass, read-only except through its own
in-place operators and item assignment, which record the time of every
change of the underlying buffer.  Its k-d tree is built on the GPU the first
time it is needed and rebuilt whenever the buffer changed after the last
build (``_update_kd_tree``).  ``nbhds`` answers exactly like
``kdtree._query`` on that tree; ``NBHDS`` returns a lazy neighbourhood
expression that evaluates in chunks; ``nbhds_dense`` gives the dense
(indices, counts) form without building per-query lists.
"""
import time

import numpy as np

from . import kdtree

__all__ = ["Points", "points", "nbhds_op"]


class Points(np.ndarray):
    _last_modified = {}

    def __new__(cls, *args, **kwargs):
        return super().__new__(cls, *args, **kwargs)

    def __array_finalize__(self, obj):
        self._last_updated = None
        self._tree = None
        if obj is not None and not isinstance(obj, Points):
            raise TypeError("Detected attempt at creating Points-type view on non-Points object.")
        base = self.__array_interface__["data"][0]
        if obj is None or base < obj._memloc or base >= obj._memloc + obj._memsize:
            # a new buffer (construction or copy)
            self._memsize = self.size * self.dtype.itemsize
            self._memloc = base
        else:
            # a view into obj's buffer: share its modification record
            self._memsize = obj._memsize
            self._memloc = obj._memloc

    def __init__(self, *args, **kwargs):
        self.flags.writeable = False

    def copy(self, order="C"):
        x = super().copy(order)
        x.flags.writeable = False
        return x

    def _record_modify_time(self):
        Points._last_modified[self._memloc] = time.time()

    def _update_kd_tree(self):
        """(Re)builds the device tree if the buffer changed since the last
        build; returns the build time in seconds, or None if none was needed."""
        if Points._last_modified.get(self._memloc) is None:
            Points._last_modified[self._memloc] = time.time()
        if self._last_updated is None or self._last_updated <= Points._last_modified[self._memloc]:
            t0 = time.time()
            self._tree = kdtree._build(np.ascontiguousarray(self.view(np.ndarray)))
            self._last_updated = time.time()
            return self._last_updated - t0
        return None

    def nbhds(self, queries=None, k=1, r=None, verbose=False):
        """Neighbourhoods as kdtree._query returns them (a list of index
        arrays): k nearest within r, or every point within r when k=None."""
        self._update_kd_tree()
        return kdtree._query(self._tree, queries=queries, k=k, dmax=r)

    def nbhds_dense(self, queries=None, k=1, r=None):
        """kNN neighbourhoods in dense form: (indices m x k, -1 padded;
        counts m)."""
        self._update_kd_tree()
        return kdtree.knn(self._tree, queries, k=k, dmax=np.inf if r is None else r)

    def NBHDS(self, queries=None, k=1, r=None, verbose=False):
        return nbhds_op(self, queries, k, r)

    def _guard(self, f):
        def guarded(*args, **kwargs):
            if self.base is not None and isinstance(self.base, np.ndarray):
                self.base.flags.writeable = True
            self.flags.writeable = True
            try:
                return f(*args, **kwargs)
            finally:
                self.flags.writeable = False
                if self.base is not None and isinstance(self.base, np.ndarray):
                    self.base.flags.writeable = False
                self._record_modify_time()
        return guarded

    def __setitem__(self, key, value):
        return self._guard(super().__setitem__)(key, value)

    def __delitem__(self, key):
        return self._guard(super().__delitem__)(key)


def _inplace(name):
    def op(self, other):
        return self._guard(getattr(np.ndarray, name).__get__(self))(other)
    op.__name__ = name
    return op


for _name in ("__iadd__", "__isub__", "__imul__", "__itruediv__", "__ifloordiv__", "__imod__", "__ipow__",
              "__ilshift__", "__irshift__", "__iand__", "__ixor__", "__ior__"):
    setattr(Points, _name, _inplace(_name))


def points(object, dtype=None, copy=True):
    """A Points copy of `object` (or a Points view of an ndarray when
    copy=False and no conversion is needed)."""
    if not copy and isinstance(object, np.ndarray) and (dtype is None or dtype == object.dtype):
        return object.view(Points)
    temp = np.asarray(object, dtype=dtype)
    ret = Points(shape=temp.shape, dtype=temp.dtype)
    ret[:] = temp
    return ret


class nbhds_op:
    """Lazy neighbourhoods of a Points object (expr.py:397-424): len() is the
    number of queries; evaluate() (or _evaluate_chunk) runs the query on the
    cached device tree."""

    def __init__(self, data, queries, k, r):
        self.data = data
        self.queries = queries
        self.k = k
        self.r = r

    def __len__(self):
        return self.data.shape[0] if self.queries is None else len(self.queries)

    def _evaluate_chunk(self, index, size, use_cache=False):
        self.data._update_kd_tree()
        if self.queries is None:
            q = np.arange(index, index + size)
        else:
            q = self.queries[index:index + size]
        return kdtree._query(self.data._tree, q, self.k, self.r)

    def evaluate(self, chunk=1_000_000):
        out = []
        for i in range(0, len(self), chunk):
            out.extend(self._evaluate_chunk(i, min(chunk, len(self) - i)))
        return out
