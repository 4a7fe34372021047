"""Autotuner for the traversal settings of a workload.

Two settings shape every kNN / normal traversal:

* the leaf bucket size of the traversal hierarchy (``set_bucket`` on a tree
  or forest): larger buckets mean fewer node visits and more candidates;
* ``lane_span`` (``pptkg_tune_set``): warps whose 32 queries span more tree
  positions than this walk the tree per lane instead of as one packet.

``tune`` times a caller-supplied workload on a sample for every combination,
keeps the fastest and leaves it applied.  The kernels' k-tiling (the
compile-time top-k capacity 4/8/16/32/64 chosen as the smallest that holds
k) is fixed, since a larger capacity only costs registers.
"""
import itertools
import time

from . import _native as N

BUCKETS = (16, 32, 64, 128)
LANE_SPANS = (-1, 64, 256, 1024)


def tune(run, set_bucket=None, buckets=BUCKETS, lane_spans=LANE_SPANS, repeats=2, sync=None):
    """Sweeps bucket x lane_span over run() (a callable doing the sample
    workload), timing the best of `repeats` runs after one warm-up run each.
    set_bucket(b) applies a bucket size (None: bucket not tuned).  sync()
    waits for the device (default: torch.cuda.synchronize).  Returns a dict
    with the chosen bucket and lane_span, their time and the whole table;
    the chosen setting stays applied."""
    if sync is None:
        import torch
        sync = torch.cuda.synchronize
    if set_bucket is None:
        buckets = (None,)
    table = []
    for b, ls in itertools.product(buckets, lane_spans):
        if b is not None:
            set_bucket(b)
        N.tune_set("lane_span", ls)
        run()
        sync()
        best = float("inf")
        for _ in range(max(1, repeats)):
            t0 = time.perf_counter()
            run()
            sync()
            best = min(best, time.perf_counter() - t0)
        table.append({"bucket": b, "lane_span": ls, "seconds": best})
    win = min(table, key=lambda r: r["seconds"])
    if win["bucket"] is not None:
        set_bucket(win["bucket"])
    N.tune_set("lane_span", win["lane_span"])
    return {"bucket": win["bucket"], "lane_span": win["lane_span"], "seconds": win["seconds"], "table": table}
