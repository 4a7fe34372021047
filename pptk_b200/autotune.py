"""Autotuner for the traversal settings of a workload.

Five settings shape every kNN / normal traversal; none changes a result:

* the leaf bucket size of the traversal hierarchy (``set_bucket`` on a tree
  or forest): larger buckets mean fewer node visits and more candidates;
* ``lane_span`` (``pptkg_tune_set``): warps whose 32 queries span more tree
  positions than this walk the tree one query per lane instead of as one
  32-query packet -- the warps-per-query choice of the kNN walks;
* ``warm_bound``: whether the warm-started lists also take the seed bound of
  a wider window of tree-order neighbours;
* ``topk_min``: the k-tiling of the register top-k lists (their compile-time
  capacity, at least the smallest of 4/8/16/32/64 that holds k);
* ``warm_mult``: the width of the warm-start window of full-capacity float
  lists, in multiples of k (2 is best for queries in tree order; 3 was
  faster for scattered kNN queries on the 20M scene).

``tune`` times a caller-supplied workload on a sample: the full grid of
bucket x lane_span first, then one pass over each further knob with the
others held at their best, keeps the fastest and leaves it applied.
"""
import itertools
import time

from . import _native as N

BUCKETS = (16, 32, 64, 128)
LANE_SPANS = (-1, 64, 256, 1024)
EXTRA_KNOBS = {"warm_bound": (0, 1), "topk_min": (0, 32), "warm_mult": (2, 3)}


def _time(run, sync, repeats):
    run()
    sync()
    best = float("inf")
    for _ in range(max(1, repeats)):
        t0 = time.perf_counter()
        run()
        sync()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(run, set_bucket=None, buckets=BUCKETS, lane_spans=LANE_SPANS, repeats=2, sync=None, extra=None):
    """Sweeps bucket x lane_span over run() (a callable doing the sample
    workload), timing the best of `repeats` runs after one warm-up run each,
    then each knob of `extra` ({name: values}; default EXTRA_KNOBS, {} for
    none) in turn.  set_bucket(b) applies a bucket size (None: bucket not
    tuned).  sync() waits for the device (default:
    torch.cuda.synchronize).  Returns a dict with the chosen settings, their
    time and the tables; the chosen settings stay applied."""
    if sync is None:
        import torch
        sync = torch.cuda.synchronize
    if set_bucket is None:
        buckets = (None,)
    extra = EXTRA_KNOBS if extra is None else extra
    table = []
    for b, ls in itertools.product(buckets, lane_spans):
        if b is not None:
            set_bucket(b)
        N.tune_set("lane_span", ls)
        table.append({"bucket": b, "lane_span": ls, "seconds": _time(run, sync, repeats)})
    win = min(table, key=lambda r: r["seconds"])
    if win["bucket"] is not None:
        set_bucket(win["bucket"])
    N.tune_set("lane_span", win["lane_span"])
    out = {"bucket": win["bucket"], "lane_span": win["lane_span"], "seconds": win["seconds"], "table": table,
           "knob_table": []}
    for name, values in extra.items():
        rows = []
        for v in values:
            N.tune_set(name, v)
            rows.append({name: v, "seconds": _time(run, sync, repeats)})
        best = min(rows, key=lambda r: r["seconds"])
        N.tune_set(name, best[name])
        out[name] = best[name]
        out["seconds"] = min(out["seconds"], best["seconds"])
        out["knob_table"].extend(rows)
    return out
