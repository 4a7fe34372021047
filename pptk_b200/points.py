"""Points with a cached device k-d tree: the hot-path callers of pptk's
``_query`` (pptk/points/points.py:87-181 for the class, expr.py:397-424 for
the lazy neighbourhood operator).

Design.  Every memory buffer that Points arrays live in has one
``_Generation`` record, shared by all Points views of that buffer.  Points
are read-only to plain numpy writes; their own writers (item assignment and
the in-place operators) unlock the buffer for the duration of the write and
then advance the record's generation number.  A Points object keeps the
device tree it built last, tagged with the generation it was built at;
``_update_kd_tree`` rebuilds exactly when the generation moved on.  The
observable behaviour is the reference's (a tree follows every write made
through any view of the buffer, and nothing is rebuilt otherwise), without
wall-clock timestamps: two writes in the same clock tick cannot be missed.

``nbhds`` answers exactly like ``kdtree._query`` on the current tree;
``NBHDS`` returns a lazy neighbourhood expression that evaluates in chunks;
``nbhds_dense`` gives the dense (indices, counts) form without building
per-query lists.
"""
import time

import numpy as np

from . import kdtree

__all__ = ["Points", "points", "nbhds_op", "zeros", "ones", "empty", "zeros_like", "ones_like", "empty_like",
           "rand", "load"]


class _Generation:
    """Write counter of one buffer: [lo, hi) are its byte addresses."""
    __slots__ = ("lo", "hi", "value")

    def __init__(self, lo, nbytes):
        self.lo, self.hi, self.value = lo, lo + nbytes, 0

    def covers(self, addr):
        return self.lo <= addr < self.hi


def _address(a):
    return a.__array_interface__["data"][0]


class Points(np.ndarray):
    """An (n, dim) point array whose k-d tree lives on the GPU and follows
    the array's contents.  Plain numpy writes are refused (the array is not
    writeable); item assignment and in-place arithmetic on the Points object
    itself are allowed and mark the buffer as changed."""

    def __array_finalize__(self, parent):
        self._tree = None
        self._tree_generation = -1
        if parent is not None and not isinstance(parent, Points):
            # ndarray.view(Points): a plain array cannot report its writes
            raise TypeError("a Points view can only be taken of a Points array; use points(a) to make a copy")
        addr = _address(self)
        gen = getattr(parent, "_gen", None)
        if gen is not None and gen.covers(addr):
            self._gen = gen  # a slice or view: the same buffer, the same counter
        else:
            self._gen = _Generation(addr, self.nbytes)  # a new buffer (construction, copy, ufunc output)

    def __init__(self, *args, **kwargs):
        self.flags.writeable = False

    def copy(self, order="C"):
        out = super().copy(order)
        out.flags.writeable = False
        return out

    # -------------------------------------------------------------- writes --
    def _owner(self):
        b = self.base
        return b if isinstance(b, np.ndarray) else None

    def _write(self, fn, *args):
        """Runs a write with the buffer unlocked, then advances its
        generation (also when the write raised part way)."""
        owner = self._owner()
        if owner is not None:
            owner.flags.writeable = True
        self.flags.writeable = True
        try:
            return fn(*args)
        finally:
            self.flags.writeable = False
            if owner is not None:
                owner.flags.writeable = False
            self._gen.value += 1

    def __setitem__(self, key, value):
        self._write(super().__setitem__, key, value)

    # -------------------------------------------------------------- trees --
    def _update_kd_tree(self):
        """Builds the device tree if none exists or the buffer was written
        since the last build; returns the build time in seconds, or None
        when the cached tree is current."""
        if self._tree is not None and self._tree_generation == self._gen.value:
            return None
        gen = self._gen.value
        t0 = time.perf_counter()
        self._tree = kdtree._build(np.ascontiguousarray(self.view(np.ndarray)))
        self._tree_generation = gen
        return time.perf_counter() - t0

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


def _inplace(name):
    base = getattr(np.ndarray, name)

    def op(self, other):
        return self._write(base, self, other)

    op.__name__ = name
    op.__doc__ = f"In-place {name[3:-2]} that marks the buffer as changed."
    return op


# += -= *= /= //= %= **= <<= >>= &= ^= |= and @= all go through _write
for _name in ("__iadd__", "__isub__", "__imul__", "__itruediv__", "__ifloordiv__", "__imod__", "__ipow__",
              "__ilshift__", "__irshift__", "__iand__", "__ixor__", "__ior__", "__imatmul__"):
    setattr(Points, _name, _inplace(_name))


# ------------------------------------------------------------ construction --
def empty(shape, dtype=float):
    return Points(shape=shape, dtype=dtype)


def zeros(shape, dtype=float):
    out = empty(shape, dtype)
    out[...] = 0
    return out


def ones(shape, dtype=float):
    out = empty(shape, dtype)
    out[...] = 1
    return out


def empty_like(a, dtype=None):
    return zeros(np.shape(a), a.dtype if dtype is None else dtype)


def zeros_like(a, dtype=None):
    return zeros(np.shape(a), a.dtype if dtype is None else dtype)


def ones_like(a, dtype=None):
    return ones(np.shape(a), a.dtype if dtype is None else dtype)


def rand(*dims):
    out = empty(dims, float)
    out[...] = np.random.rand(*dims)
    return out


def points(object, dtype=None, copy=True):
    """A Points copy of `object`.  With copy=False a Points array is
    returned as a view of itself when no conversion is needed."""
    if not copy and isinstance(object, Points) and (dtype is None or dtype == object.dtype):
        return object.view(Points)
    src = np.asarray(object, dtype=dtype)
    out = empty(src.shape, src.dtype)
    out[...] = src
    return out


def load(file, **kwargs):
    """numpy.load into a Points array."""
    return points(np.load(file, **kwargs))


class nbhds_op:
    """Lazy neighbourhoods of a Points object (expr.py:397-424): len() is the
    number of queries; evaluate() (or _evaluate_chunk) runs the query on the
    object's current device tree."""

    def __init__(self, data, queries, k, r):
        self.data = data
        self.queries = queries
        self.k = k
        self.r = r

    def __len__(self):
        return self.data.shape[0] if self.queries is None else len(self.queries)

    def _evaluate_chunk(self, index, size, use_cache=False):
        self.data._update_kd_tree()
        q = np.arange(index, index + size) if self.queries is None else self.queries[index:index + size]
        return kdtree._query(self.data._tree, q, self.k, self.r)

    def evaluate(self, chunk=1_000_000):
        out = []
        for i in range(0, len(self), chunk):
            out.extend(self._evaluate_chunk(i, min(chunk, len(self) - i)))
        return out
