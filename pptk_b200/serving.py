"""Continuous-batching server for resident k-d trees.

Trees built through the server stay in HBM.  Build, kNN, r-near and normal
requests of very different sizes are admitted first-in first-out against an
HBM budget; whenever an execution slot frees up, every admitted query request
is folded into the next batch -- kNN requests (same k, dmax, query dtype)
across all trees become one multi-tree launch, normal requests likewise --
and the batch runs on that slot's CUDA stream while other slots keep
running.  A request's answer does not depend on what it was batched with:
the multi-tree kernels give every query exactly the result it gets alone.

The engine that executes batches is pluggable (``GpuEngine`` by default), so
the scheduling logic can be exercised without a GPU.
"""
import math
import threading
import time
from collections import deque
from concurrent.futures import Future, ThreadPoolExecutor

import numpy as np

# Bytes per point of a resident tree (tree-ordered points with index 16 B,
# forward map 4 B, build records and traversal nodes ~48 B) and of a build's
# transient scratch; bytes per query of a batch.
TREE_BYTES_PER_POINT = 72
BUILD_SCRATCH_PER_POINT = 160
QUERY_BYTES = 96


def _kclass(k):
    """Top-k capacity class of k (the kernels' compile-time capacities)."""
    for c in (4, 8, 16, 32, 64):
        if k <= c:
            return c
    return k


def _first_k(idx, cnt, k, k_launch):
    """The result of a k-query taken from a k_launch-query (k <= k_launch):
    the first k columns and the counts capped at k."""
    if k == k_launch:
        return idx, cnt
    if isinstance(cnt, np.ndarray):
        return idx[:, :k], np.minimum(cnt, k)
    return idx[:, :k], cnt.clamp(max=k)


class Request:
    __slots__ = ("kind", "args", "future", "t_submit", "t_start", "t_done", "bytes", "m", "key", "next_row",
                 "rows_done", "parts")

    def __init__(self, kind, args, nbytes, m, key=None):
        self.kind = kind
        self.args = args
        self.future = Future()
        self.t_submit = time.perf_counter()
        self.t_start = None
        self.t_done = None
        self.bytes = nbytes
        self.m = m
        self.key = key


class GpuEngine:
    """Executes batches with the native library on one device."""

    def __init__(self, device=0):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)

    def stream(self, high_priority=False):
        """A CUDA stream of this device; high-priority streams get free SMs
        first, so a small batch does not wait behind a large one."""
        lo, hi = self.torch.cuda.Stream.priority_range()
        return self.torch.cuda.Stream(device=self.device, priority=hi if high_priority else lo)

    def build(self, points, maxleafsize, emptysplit, stream):
        from . import kdtree
        with self.torch.cuda.stream(stream):
            return kdtree._build(points, maxleafsize=maxleafsize, emptysplit=emptysplit)

    @staticmethod
    def _merge(trees, parts):
        """Requests on the same tree become one group of the launch: returns
        the distinct trees, each one's concatenated parts, and for every
        request its (group, first row, rows)."""
        order, where = {}, []
        for t, x in zip(trees, parts):
            g = order.setdefault(id(t), len(order))
            where.append(g)
        uniq = [None] * len(order)
        groups = [[] for _ in order]
        for t, x, g in zip(trees, parts, where):
            uniq[g] = t
            groups[g].append(x)
        lens = [[len(x) for x in grp] for grp in groups]
        starts = np.concatenate([[0], np.cumsum([sum(l) for l in lens])]).astype(np.int64)
        cursor = [int(starts[g]) for g in range(len(uniq))]
        spans = []
        for x, g in zip(parts, where):
            spans.append((cursor[g], len(x)))
            cursor[g] += len(x)
        return uniq, groups, starts, spans

    def _to_host(self, tensors):
        """Pinned host copies on the current stream (complete once the
        stream is synchronised), as numpy arrays."""
        out = []
        for t in tensors:
            h = self.torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            h.copy_(t, non_blocking=True)
            out.append(h.numpy())
        return out

    def knn_batch(self, trees, queries, k, dmax, stream, host=False):
        """queries: list of per-request query arrays (numpy or CUDA tensors);
        requests on the same tree share one group of the launch.  host: the
        results come back as numpy arrays (copied on this stream)."""
        import ctypes
        from . import _native as N
        torch = self.torch
        with torch.cuda.stream(stream):
            qs = [torch.as_tensor(q, device=self.device) for q in queries]
            dt = qs[0].dtype if qs[0].dtype in (torch.float32, torch.float64) else torch.float64
            uniq, groups, rows, spans = self._merge(trees, qs)
            q = torch.cat([x.to(dt) for grp in groups for x in grp]).contiguous()
            m = int(rows[-1])
            idx = torch.empty((m, k), dtype=torch.int32, device=self.device)
            cnt = torch.empty((m,), dtype=torch.int32, device=self.device)
            handles = (ctypes.c_void_p * len(uniq))(*[t._h.value for t in uniq])
            N.call("pptkg_multi_knn", handles, len(uniq), N.ptr(q), N.ptr(rows), 0 if dt == torch.float32 else 1,
                   N.MEM_DEVICE, int(k), float(np.float32(dmax)), N.ptr(idx), N.ptr(cnt),
                   ctypes.c_void_p(stream.cuda_stream), where="serving knn")
            if host:
                idx, cnt = self._to_host([idx, cnt])
        return [(idx[a:a + n], cnt[a:a + n]) for a, n in spans]

    def normals_batch(self, trees, indices, k, r, precision, stream, host=False):
        import ctypes
        from . import _native as N
        from .estimate_normals import PRECISIONS
        torch = self.torch
        with torch.cuda.stream(stream):
            ids = []
            for t, ix in zip(trees, indices):
                if ix is None:
                    ix = RowRange(0, t.n)
                if isinstance(ix, RowRange):
                    ix = torch.arange(ix.lo, ix.hi, dtype=torch.int32, device=self.device)
                ids.append(torch.as_tensor(ix, device=self.device).to(torch.int32))
            uniq, groups, rows, spans = self._merge(trees, ids)
            q = torch.cat([x for grp in groups for x in grp]).contiguous()
            m = int(rows[-1])
            tdt = torch.float32 if trees[0].dtype == np.float32 else torch.float64
            ev = torch.empty((m, 3), dtype=tdt, device=self.device)
            handles = (ctypes.c_void_p * len(uniq))(*[t._h.value for t in uniq])
            N.call("pptkg_multi_normals", handles, len(uniq), N.ptr(q), N.ptr(rows), N.MEM_DEVICE, int(k),
                   ctypes.c_float(float(np.float32(r))), 1, PRECISIONS[precision], N.ptr(ev), None, None,
                   ctypes.c_void_p(stream.cuda_stream), where="serving normals")
            if host:
                ev, = self._to_host([ev])
        return [ev[a:a + n] for a, n in spans]

    def rnear(self, tree, queries, dmax, stream, host=False):
        from . import kdtree
        with self.torch.cuda.stream(stream):
            q = self.torch.as_tensor(queries, device=self.device)
            off, hits = kdtree.rnear(tree, q, dmax)
            if host:
                return off.cpu().numpy(), hits.cpu().numpy()
            return off, hits

    def synchronize(self, stream):
        stream.synchronize()

    def mark(self, stream):
        """A timing event recorded on `stream` at this point of its work."""
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e


class _Slice:
    """Rows [lo, hi) of a request, the unit that batches are made of."""
    __slots__ = ("r", "lo", "hi")

    def __init__(self, r, lo, hi):
        self.r, self.lo, self.hi = r, lo, hi

    @property
    def m(self):
        return self.hi - self.lo


class RowRange:
    """Rows lo .. hi-1 of a tree's input, standing for a normal request over
    all rows (indices None) cut into slices."""
    __slots__ = ("lo", "hi")

    def __init__(self, lo, hi):
        self.lo, self.hi = lo, hi

    def __len__(self):
        return self.hi - self.lo


def _rows(x, lo, hi):
    if isinstance(x, RowRange):
        return RowRange(x.lo + lo, x.lo + hi)
    return x[lo:hi]


def _concat(parts):
    """Joins the per-slice results of one request (numpy arrays or CUDA
    tensors, or tuples of them) along the query rows."""
    if len(parts) == 1:
        return parts[0]
    if isinstance(parts[0], tuple):
        return tuple(_concat([p[i] for p in parts]) for i in range(len(parts[0])))
    if isinstance(parts[0], np.ndarray):
        return np.concatenate(parts)
    import torch
    return torch.cat(parts)


class Server:
    """Continuous-batching server.

    budget_bytes: HBM the server may commit to resident trees plus the
        transient needs of admitted requests.
    slots: batches that may run at once, each on its own CUDA stream.  The
        last `fast_slots` of them run on high-priority streams and serve
        small requests only (at most `small_batch` queries each), taken from
        anywhere in the queue, so that a small request never waits behind a
        large one.
    max_batch_queries: upper bound on the queries folded into one batch; a
        request larger than the cap runs in cap-sized slices, so requests
        submitted after it interleave with its slices.
    batch_ms: optional time budget of one batch: the cap becomes the measured
        rate (queries per second of recent batches) times this budget, within
        [min_batch_queries, max_batch_queries].
    max_host_batch_queries: the upper bound for batches that return numpy
        results.  Smaller batches let one batch's host copies overlap more
        of another batch's kernels, but each pays its own copies and
        launches: on the 20M scene the end-to-end rate with numpy requests
        was 267 / 297 / 375 M queries/s at caps of 4M / 8M / 20M, so the
        default is the batch cap itself.

    defer_ms: while a normal-slot batch is running, another normal slot
        starts a batch only once at least min_batch_queries queries wait or
        the oldest waiting request has waited defer_ms (0: start at once).
        Under steady arrivals this folds the requests that arrive during a
        batch into the next one instead of a string of small batches, which
        run at a lower query rate (less coherent query packets, fixed costs
        per batch).  The defaults (15 ms, 4M queries) gave the steadiest
        tail of the policies measured on the 20M-point scene under Poisson
        arrivals at half the burst throughput.
    trace: keep, for every batch, CUDA events recorded on its stream before
        and after its work (``trace`` list of (kinds, fast slot, start,
        end)), so that the device-side overlap of batches can be checked.

    Requests are admitted first-in first-out (the fast slots excepted)
    against the HBM budget; a request's Future may be cancelled (``future.cancel()``) until its last
    rows are answered: rows not yet started are never run, and the answer of
    rows in flight is discarded.  A batch that fails fails the requests it
    held rows of; the server keeps serving.
    """

    def __init__(self, budget_bytes=150e9, slots=3, device=0, max_batch_queries=20_000_000, engine=None,
                 fast_slots=1, small_batch=65_536, max_host_batch_queries=20_000_000, batch_ms=None,
                 min_batch_queries=4_000_000, trace=False, defer_ms=15.0):
        self.budget = float(budget_bytes)
        self.engine = engine or GpuEngine(device)
        self.max_batch = int(max_batch_queries)
        self.max_host_batch = int(max_host_batch_queries)
        self.small_batch = int(small_batch)
        self.batch_ms = None if batch_ms is None else float(batch_ms)
        self.min_batch = int(min_batch_queries)
        self.defer_s = max(0.0, float(defer_ms)) / 1e3
        self._normal_running = 0
        self._rate = None  # queries per second of recent batches (EMA)
        self.trace = [] if trace else None
        self.trees = {}
        self.tree_bytes = {}
        self._next_id = 0
        self._queue = deque()
        self._committed = 0.0
        self._cv = threading.Condition()
        fast_slots = max(0, min(int(fast_slots), slots - 1))
        self._free = [(self.engine.stream(False), False) for _ in range(slots - fast_slots)]
        self._free += [(self.engine.stream(True), True) for _ in range(fast_slots)]
        self._pool = ThreadPoolExecutor(max_workers=slots, thread_name_prefix="pptk-b200-slot")
        self._running = True
        self._done = []
        self._batches = 0
        self._thread = threading.Thread(target=self._loop, name="pptk-b200-server", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------ requests --
    def build(self, points, maxleafsize=10, emptysplit=0.2):
        """Future of a tree id."""
        n = int(points.shape[0])
        r = Request("build", (points, maxleafsize, emptysplit), n * (TREE_BYTES_PER_POINT + BUILD_SCRATCH_PER_POINT), n)
        return self._submit(r)

    def knn(self, tree_id, queries, k=1, dmax=math.inf, to_host=None):
        """Future of (indices m x k, counts m) for point queries.  to_host:
        numpy results (default: when the queries are a numpy array),
        otherwise CUDA tensors."""
        m = int(queries.shape[0])
        dt = str(getattr(queries, "dtype", "float64"))
        host = isinstance(queries, np.ndarray) if to_host is None else bool(to_host)
        k = int(k)
        if k < 1:
            raise ValueError("k must be positive")
        # requests whose k share a top-k capacity class run as one launch at
        # the class's largest k; each gets its first k columns (the exact
        # top-k of its own query)
        r = Request("knn", (tree_id, queries, k), m * (QUERY_BYTES + 4 * _kclass(k)), m,
                    key=("knn", _kclass(k), float(dmax), dt, host))
        return self._submit(r)

    def normals(self, tree_id, indices=None, k=16, r=math.inf, precision="auto", to_host=None):
        """Future of the normals (m x 3) of the tree's input rows `indices`
        (all rows when None), over k nearest neighbours within r.  to_host
        as for knn (default: when the indices are a numpy array)."""
        host = isinstance(indices, np.ndarray) if to_host is None else bool(to_host)
        if indices is None:
            tree = self.trees.get(tree_id)
            if tree is None:
                f = Future()
                f.set_exception(KeyError(f"unknown tree {tree_id}"))
                return f
            indices = RowRange(0, tree.n)
        m = int(len(indices))
        req = Request("normals", (tree_id, indices), m * (QUERY_BYTES + 4 * int(k)), m,
                      key=("normals", int(k), float(r), precision, host))
        return self._submit(req)

    def rnear(self, tree_id, queries, dmax, to_host=None):
        """Future of (offsets m + 1, hits) of the points within dmax of each
        query point, in the reference's order.  to_host as for knn (default:
        numpy results when the queries are a numpy array)."""
        m = int(queries.shape[0])
        host = isinstance(queries, np.ndarray) if to_host is None else bool(to_host)
        return self._submit(Request("rnear", (tree_id, queries, float(dmax), host), m * QUERY_BYTES * 8, m))

    def drop(self, tree_id):
        """Releases a resident tree."""
        with self._cv:
            self.trees.pop(tree_id, None)
            self._committed -= self.tree_bytes.pop(tree_id, 0)
            self._cv.notify_all()

    def _submit(self, r):
        if r.bytes > self.budget:
            r.future.set_exception(MemoryError(f"request needs {r.bytes:.3g} B, above the budget {self.budget:.3g} B"))
            return r.future
        r.next_row = 0
        r.rows_done = 0
        r.parts = {}
        with self._cv:
            if not self._running:
                raise RuntimeError("server closed")
            self._queue.append(r)
            self._cv.notify_all()
        return r.future

    # ----------------------------------------------------------- scheduler --
    def batch_cap(self, host=False):
        """Queries a kNN / normal batch may hold now."""
        top = min(self.max_host_batch, self.max_batch) if host else self.max_batch
        if self.batch_ms is None or self._rate is None:
            return top
        return int(min(top, max(self.min_batch, self._rate * self.batch_ms / 1e3)))

    def _admit(self, fast):
        """Slices of requests for the next batch, under the HBM budget.

        A normal slot takes requests first-in first-out from the head of
        the queue and folds kNN / normal requests up to the batch cap; a
        request never straddles two batches unless it is larger than the cap
        by itself, in which case it runs in cap-sized slices, one batch each.
        A fast slot takes small requests (at most small_batch queries) from
        anywhere in the queue, oldest first, up to small_batch queries in
        all, so that a small request never waits behind a large one.  A
        build or r-near request runs as a batch of its own."""
        out = []
        queries = 0
        host = False
        q = self._queue
        i = 0
        while i < len(q):
            r = q[i]
            if r.future.done():  # cancelled (or failed) while queued: its rows
                del q[i]         # not yet admitted never run (nothing of them was committed)
                continue
            if r.kind != "build" and r.args[0] not in self.trees:
                del q[i]
                r.future.set_exception(KeyError(f"unknown tree {r.args[0]}"))
                continue
            small = r.kind != "build" and r.m <= self.small_batch and r.next_row == 0
            if fast and not small:
                i += 1
                continue
            exclusive = r.kind in ("build", "rnear")
            r_host = bool(r.key and r.key[-1] is True)
            cap = min(self.batch_cap(host or r_host), self.small_batch) if fast else self.batch_cap(host or r_host)
            left = r.m - r.next_row
            if out and (exclusive or queries + left > cap):
                break
            take = left if (exclusive or left <= cap) else cap
            part = r.bytes * take / max(r.m, 1) if r.m else r.bytes
            if self._committed + part > self.budget:
                break
            if r.next_row == 0:
                r.t_start = time.perf_counter()
            out.append(_Slice(r, r.next_row, r.next_row + take))
            r.next_row += take
            self._committed += part
            queries += take
            host = host or r_host
            if r.next_row >= r.m:
                del q[i]
            else:
                break  # a slice of a large request is a batch of its own
            if exclusive:
                break
        return out

    def _loop(self):
        while True:
            with self._cv:
                while self._running and (not self._queue or not self._free):
                    self._cv.wait(0.01)
                if not self._running and not self._queue:
                    return
                if not self._free:
                    continue
                batch, slot = [], None
                defer = self._defer()
                # a fast slot first when small requests wait, then the others
                for i in sorted(range(len(self._free)), key=lambda j: not self._free[j][1]):
                    if defer and not self._free[i][1]:
                        continue
                    batch = self._admit(self._free[i][1])
                    if batch:
                        slot = self._free.pop(i)
                        break
                if not batch:
                    self._cv.wait(0.001)
                    continue
                self._batches += 1
                if not slot[1]:
                    self._normal_running += 1
            self._pool.submit(self._run, batch, slot)

    def _defer(self):
        """True while a new normal-slot batch should wait (see defer_ms)."""
        if self.defer_s <= 0 or self._normal_running == 0 or not self._queue:
            return False
        waiting = 0
        oldest = None
        for r in self._queue:
            if r.kind in ("knn", "normals"):
                waiting += r.m - r.next_row
                oldest = r.t_submit if oldest is None else min(oldest, r.t_submit)
            else:
                return False  # builds and r-near run at once
        if waiting >= self.min_batch or oldest is None:
            return False
        return time.perf_counter() - oldest < self.defer_s

    def _run(self, batch, slot):
        stream = slot[0]
        t0 = time.perf_counter()
        live = [s for s in batch if not s.r.future.done()]
        marks = self.trace is not None and hasattr(self.engine, "mark")
        try:
            e0 = self.engine.mark(stream) if marks else None
            groups = {}
            for sl in live:
                r = sl.r
                groups.setdefault(r.key if r.key else (r.kind, id(r)), []).append(sl)
            for key, ss in groups.items():
                kind = ss[0].r.kind
                if kind == "build":
                    r = ss[0].r
                    tree = self.engine.build(*r.args, stream)
                    with self._cv:
                        tid = self._next_id
                        self._next_id += 1
                        self.trees[tid] = tree
                        self.tree_bytes[tid] = r.m * TREE_BYTES_PER_POINT
                        self._committed += self.tree_bytes[tid]
                    self._finish(ss, [tid], stream)
                elif kind == "knn":
                    trees = [self.trees[s.r.args[0]] for s in ss]
                    kl = max(s.r.args[2] for s in ss)
                    res = self.engine.knn_batch(trees, [_rows(s.r.args[1], s.lo, s.hi) for s in ss], kl, key[2],
                                                stream, host=key[4])
                    # (host results arrive by asynchronous copies: the counts are
                    # capped only once the stream has finished them)
                    if key[4]:
                        self.engine.synchronize(stream)
                    res = [_first_k(i, c, s.r.args[2], kl) for (i, c), s in zip(res, ss)]
                    self._finish(ss, res, stream)
                elif kind == "normals":
                    trees = [self.trees[s.r.args[0]] for s in ss]
                    res = self.engine.normals_batch(trees, [_rows(s.r.args[1], s.lo, s.hi) for s in ss], key[1],
                                                    key[2], key[3], stream, host=key[4])
                    self._finish(ss, res, stream)
                elif kind == "rnear":
                    r = ss[0].r
                    res = self.engine.rnear(self.trees[r.args[0]], r.args[1], r.args[2], stream, host=r.args[3])
                    self._finish(ss, [res], stream)
            if marks:
                e1 = self.engine.mark(stream)
                with self._cv:
                    self.trace.append((sorted({s.r.kind for s in live}), slot[1], e0, e1))
            q = sum(s.m for s in live if s.r.kind in ("knn", "normals"))
            dt = time.perf_counter() - t0
            if q >= self.min_batch // 4 and dt > 0:
                with self._cv:
                    self._rate = q / dt if self._rate is None else 0.7 * self._rate + 0.3 * (q / dt)
        except Exception as e:  # a failed batch fails its requests, not the server
            for sl in batch:
                if not sl.r.future.done():
                    sl.r.future.set_exception(e)
        finally:
            with self._cv:
                for sl in batch:
                    self._committed -= sl.r.bytes * sl.m / max(sl.r.m, 1) if sl.r.m else sl.r.bytes
                if not slot[1]:
                    self._normal_running -= 1
                self._free.append(slot)
                self._cv.notify_all()

    def _finish(self, slices, results, stream):
        self.engine.synchronize(stream)
        t = time.perf_counter()
        for sl, res in zip(slices, results):
            r = sl.r
            with self._cv:
                r.parts[sl.lo] = res
                r.rows_done += sl.m
                complete = r.rows_done >= r.m
            if not complete:
                continue
            r.t_done = t
            out = _concat([r.parts[lo] for lo in sorted(r.parts)]) if r.kind in ("knn", "normals") else res
            r.parts = {}
            with self._cv:
                self._done.append((r.kind, r.m, r.t_submit, r.t_done))
            if not r.future.done():
                try:
                    r.future.set_result(out)
                except Exception:  # cancelled meanwhile
                    pass

    # --------------------------------------------------------------- info --
    def stats(self, since=0.0):
        """Per-kind request count, queries, p50/p99 latency (s) and queries/s
        over the requests finished after `since` (perf_counter time)."""
        with self._cv:
            done = [d for d in self._done if d[3] >= since]
        out = {}
        for kind in sorted({d[0] for d in done}):
            ds = [d for d in done if d[0] == kind]
            lat = np.array([d[3] - d[2] for d in ds])
            q = sum(d[1] for d in ds)
            span = max(d[3] for d in ds) - min(d[2] for d in ds)
            out[kind] = {"requests": len(ds), "queries": q, "p50_s": float(np.percentile(lat, 50)),
                         "p99_s": float(np.percentile(lat, 99)), "queries_per_s": q / span if span > 0 else None}
        out["batches"] = self._batches
        return out

    def close(self):
        """Stops admitting work: requests still queued fail with
        RuntimeError, running batches finish."""
        with self._cv:
            self._running = False
            while self._queue:
                r = self._queue.popleft()
                if not r.future.done():
                    r.future.set_exception(RuntimeError("server closed"))
            self._cv.notify_all()
        self._thread.join()
        self._pool.shutdown(wait=True)
