"""Benchmark of the pptk hot path on B200: kNN + normal queries per second at
k=16 on the 20M-point scene, plain per-call drop-in vs batched serving.

Workload (default ``--workload serving``): a 20M-point float32 lidar-like
scene (pptk_b200.synth.lidar_scene, seed 2) whose k-d tree is resident in
HBM, and a seeded request stream over it (pptk_b200.synth.request_mix):
alternating kNN requests (k=16, the coordinates of random scene points as
query points) and normal requests (k=16, r=inf, random scene rows), query
counts log-uniform in [1k, 1M], 20M queries of each kind.  One step answers
the whole stream (40M queries).

* ``value``: the serving form (pptk_b200.serving.Server: continuous
  batching over CUDA streams, requests on one tree merged per launch),
  request inputs and results resident in HBM; timed with CUDA events around
  the step after a device synchronisation on both sides.
* ``plain``: the same requests, one drop-in call each, as a pptk user makes
  them: ``kdtree.knn(tree, points, 16)`` on a tree built once and
  ``estimate_normals(points, 16, inf, subsample=rows)`` (which builds its own
  tree on every call, as the reference does); device inputs, and host numpy
  inputs for ``plain.e2e``.  Timed on a bounded sample of the stream.
* ``latency``: p50/p99 request latency of the server under Poisson arrivals
  at half of the measured serving throughput (``latency_at_quarter_load``:
  at a quarter), and of the plain calls.
* ``e2e``: the serving form through its public API with pinned host numpy
  inputs and numpy results (host<->device copies inside the timed region).
* ``roofline``: the fused kNN+PCA normal kernel's algorithmic bytes (216 B
  per query) over its measured time inside the step, against the measured
  HBM copy bandwidth.
* ``cpu_baseline``: the reference's own k-d tree (compiled from its sources
  in oracle/_ref), built once over the same 20M-point scene (serial build,
  reported separately as ``build_s``), answering a bounded random sample of
  the same request stream's rows -- kNN k=16 point queries and normal
  queries (the restated normal loop over the resident tree) -- using every
  host core.  Units are the serving form's: one query is one kNN request
  row or one normal request row.
* ``precision``: angular error (p50/p99/max, radians) of the FP32 normal
  path against FP64 on three clouds (200k uniform float32 k=16, the 20M
  scene k=16, 10M float64 planar patches offset 1e5 m k=24): all rows
  against the device FP64 path, and 20k sampled rows against the CPU FP64
  oracle (float64 covariance of the oracle's own neighbours).

``--workload plain`` times one drop-in ``estimate_normals`` over all 20M
points instead (device build + fused kNN+PCA).  ``--impl reference`` times
only the CPU reference path on the same metric, config and units.
Multi-GPU (torchrun): every rank runs an independent replica (weak
scaling); there is no collective on the data path.

With one GPU the default run also measures the other configurations
briefly (``configs``: the scene's kNN k=32 and r-near r=0.5 m, the 4,096-
cloud ragged batch, the 64-tree serving mix) with 3 warm-up and at most 5
timed steps each.  Bulky per-stage data is printed on ``{"detail": ...}``
lines before the final JSON line, which keeps the headline figures.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "kNN+normal queries/s at k=16 on 20M pts (plain vs batched/serving); p50/p99 lat"
BYTES_PER_QUERY = 216  # 3*4 query + 16*3*4 neighbours + 3*4 normal (f32, indices not materialised)
# one walk for the self kNN and the normal (k=16, f32): 3*4 query + 16*(3*4 + 4) neighbours read,
# 16*4 indices + 4 count + 3*4 normal written
BYTES_PER_QUERY_FUSED = 12 + 16 * 16 + 64 + 4 + 12


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="serving", choices=["serving", "plain", "ragged", "multitree", "scene"])
    p.add_argument("--points", type=int, default=20_000_000)
    p.add_argument("--k", type=int, default=16)
    p.add_argument("--slots", type=int, default=3)
    p.add_argument("--max-batch", type=int, default=20_000_000, help="queries folded into one server batch")
    p.add_argument("--batch-ms", type=float, default=None,
                   help="time budget of one server batch (None: batches capped by --max-batch only)")
    p.add_argument("--max-host-batch", type=int, default=20_000_000,
                   help="queries folded into one server batch that returns numpy results")
    p.add_argument("--plain-sample", type=int, default=24, help="requests timed through the plain calls")
    p.add_argument("--latency-seconds", type=float, default=3.0)
    p.add_argument("--cpu-sample", type=int, default=1_000_000,
                   help="request rows (half kNN, half normals) per timed CPU-reference sample")
    p.add_argument("--configs", default="scene,ragged,multitree",
                   help="other configurations measured after the default workload (1 GPU; '' for none)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-precision", action="store_true", help="skip the FP32-vs-FP64 angular error report")
    p.add_argument("--clouds", type=int, default=4096, help="ragged workload: clouds in the batch")
    p.add_argument("--no-autotune", action="store_true",
                   help="ragged workload: keep the default traversal settings (for profiling runs)")
    p.add_argument("--tune", action="append", default=[], metavar="NAME=VALUE",
                   help="a traversal knob applied before the run (pptkg_tune_set), e.g. lane_span=64")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_reference(points, k, sample, seed=0):
    """Times the reference tree + restated normal loop on a sample of the
    workload with all host threads; returns (queries/s, threads, seconds)."""
    from oracle import build_oracle
    from oracle import oracle as O
    if not O.ref_available():
        build_oracle.build_ref()
    rng = np.random.default_rng(seed)
    sel = np.sort(rng.choice(len(points), size=min(sample, len(points)), replace=False))
    P = np.ascontiguousarray(points[sel])
    threads = O.ref_lib().ref_max_threads()
    if O.ref_available():
        t0 = time.perf_counter()
        O.ref_estimate_normals(P, k, np.inf)
        dt = time.perf_counter() - t0
        kind = "reference"
    else:
        t0 = time.perf_counter()
        O.port_estimate_normals(P, k, np.inf)
        dt = time.perf_counter() - t0
        kind = "port"
    return len(P) / dt, threads, dt, kind, len(P)


def cpu_baseline_obj(pts, args):
    """CPU baseline of the plain workload: the reference's per-call
    estimate_normals (tree build included) on a sample of the scene."""
    try:
        qps, threads, dt, kind, ns = cpu_reference(pts, args.k, args.cpu_sample)
        return {"value": qps, "unit": "queries/s", "cores": threads, "kind": kind,
                "sample": f"{ns} random points of the scene: tree build + kNN k={args.k} + PCA per point "
                          f"({dt:.1f} s)"}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": "queries/s", "cores": None, "kind": "reference",
                "sample": f"unavailable: {e}"}


class RefScene:
    """The reference's own k-d tree (oracle/_ref) built once over the whole
    scene -- the resident-tree counterpart of the serving form.  The build is
    the reference's serial RecursiveBuildHelper (TBB absent), timed and
    reported on its own; queries run on every host thread."""

    def __init__(self, pts):
        from oracle import build_oracle
        from oracle import oracle as O
        if not O.ref_available():
            build_oracle.build_ref()
        self.pts = pts
        t0 = time.perf_counter()
        self.tree = O.RefTree(pts)
        self.build_s = time.perf_counter() - t0
        self.threads = O.ref_lib().ref_max_threads()

    def mix_sample(self, mix, k, sample, seed):
        """Answers `sample` rows drawn from the request stream (half from the
        kNN requests' rows, as point queries; half from the normal requests'
        rows); returns the timing of the queries alone."""
        rng = np.random.default_rng(seed)
        knn_rows = np.concatenate([r for kind, r in mix if kind == "knn"])
        norm_rows = np.concatenate([r for kind, r in mix if kind == "normals"])
        kq = knn_rows[rng.integers(0, len(knn_rows), sample // 2)]
        nq = norm_rows[rng.integers(0, len(norm_rows), sample - sample // 2)]
        Q = np.ascontiguousarray(self.pts[kq])
        t0 = time.perf_counter()
        self.tree.knn(Q, k)
        t1 = time.perf_counter()
        self.tree.normals(nq, k)
        t2 = time.perf_counter()
        return {"queries": len(kq) + len(nq), "seconds": t2 - t0, "value": (len(kq) + len(nq)) / (t2 - t0),
                "knn_queries_per_s": len(kq) / (t1 - t0), "normal_queries_per_s": len(nq) / (t2 - t1)}

    def describe(self, sample, k):
        return (f"ref tree on the {len(self.pts)}-pt scene, built once (build_s); {sample} request rows/step, half "
                f"kNN k={k}, half normals; OpenMP for TBB")


def serving_cpu_baseline(pts, mix, args):
    try:
        ref = RefScene(pts)
        r = ref.mix_sample(mix, args.k, args.cpu_sample, seed=0)
        return {"value": r["value"], "unit": "queries/s", "cores": ref.threads, "kind": "reference",
                "sample": ref.describe(args.cpu_sample, args.k), "build_s": ref.build_s,
                "knn_queries_per_s": r["knn_queries_per_s"], "normal_queries_per_s": r["normal_queries_per_s"]}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": "queries/s", "cores": None, "kind": "reference",
                "sample": f"unavailable: {e}"}


def run_reference(args):
    """The reference arm, on the default workload's metric, units and config:
    the reference tree resident over the 20M-point scene, each step a fresh
    bounded sample of the same request stream."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from pptk_b200 import synth
    pts = synth.lidar_scene(args.points, seed=2)
    mix = synth.request_mix(len(pts), len(pts), seed=11)
    ref = RefScene(pts)
    vals = []
    for i in range(args.warmup + args.steps):
        r = ref.mix_sample(mix, args.k, args.cpu_sample, seed=100 + i)
        if i >= args.warmup:
            vals.append(r)
    value = float(sum(v["queries"] for v in vals) / sum(v["seconds"] for v in vals))
    ms = float(np.mean([v["seconds"] for v in vals])) * 1e3
    knn_rate = float(np.mean([v["knn_queries_per_s"] for v in vals]))
    norm_rate = float(np.mean([v["normal_queries_per_s"] for v in vals]))
    line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"lidar_scene_{len(pts)}_f32 resident tree; rows of the kNN k={args.k} / normal "
                                   f"k={args.k} request stream (sampled {args.cpu_sample} per step)",
                       "points": len(pts), "k": args.k, "unit": "one kNN request row or one normal request row"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": ref.threads, "kind": "reference",
                             "sample": ref.describe(args.cpu_sample, args.k)},
            "build_s": ref.build_s, "knn_queries_per_s": knn_rate, "normal_queries_per_s": norm_rate,
            "plain_estimate_normals_call_s": {
                "what": "one estimate_normals call over all scene points, as the reference API does it: serial "
                        "build + the normal loop",
                "seconds": ref.build_s + len(pts) / norm_rate},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


class Ctx:
    """Per-rank plumbing: device, barrier, max over ranks, native library.
    Every rank is an independent replica; the only collectives are the
    barriers around the timed region and the max of the per-rank times.
    backend/device default to NCCL on this rank's GPU (gloo/cpu for tests
    of the replica logic)."""

    def __init__(self, backend="nccl", device=None):
        import torch
        self.torch = torch
        self.world, self.rank, self.local = dist_env()
        self.device = device or f"cuda:{self.local}"
        if self.device.startswith("cuda"):
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group(backend, timeout=timedelta(seconds=300))
        from pptk_b200 import _native as N
        self.N = N
        self.lib = N.lib()

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(self, x):
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank, seconds):
        """Whole-job rate: every rank's units over the slowest rank's time."""
        return self.world * units_per_rank / self.max_over_ranks(seconds)

    def stage(self, name):
        t, c = ctypes.c_double(), ctypes.c_int64()
        self.lib.pptkg_profile_get(name.encode(), ctypes.byref(t), ctypes.byref(c))
        return t.value, c.value

    def finish(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


def device_timed(ctx, fn, steps):
    """Runs fn `steps` times between barriers and device synchronisations,
    timed by CUDA events on the current stream; returns (ms per step,
    launches per step, clocks)."""
    torch = ctx.torch
    stream = torch.cuda.current_stream()
    clocks = ClockSampler(ctx.local)
    clocks.start()
    l0 = ctx.lib.pptkg_launch_count()
    ctx.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    torch.cuda.synchronize()
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.barrier()
    launches = (ctx.lib.pptkg_launch_count() - l0) // max(steps, 1)
    return e0.elapsed_time(e1) / steps, int(launches), clocks.stop()


class ResultSink:
    """Takes a load test's futures as a client would: each answer is checked
    (and handed to on_result) when it arrives, then dropped, so a latency run
    keeps no answers alive in HBM -- held to the end, the answers of a
    6-second run at half load (tens of GB) made every batch allocate new
    device memory, and those allocations showed up as 100-500 ms stalls."""

    def __init__(self, on_result=None):
        self.cv = threading.Condition()
        self.n = 0
        self.errors = []
        self.on_result = on_result

    def add(self, fut, tag=None):
        with self.cv:
            self.n += 1

        def done(f):
            try:
                res = f.result()
                if self.on_result is not None:
                    self.on_result(tag, res)
            except BaseException as e:  # noqa: BLE001 -- reported by wait()
                self.errors.append(e)
            with self.cv:
                self.n -= 1
                self.cv.notify_all()

        fut.add_done_callback(done)

    def wait(self):
        with self.cv:
            while self.n:
                self.cv.wait(0.1)
        if self.errors:
            raise self.errors[0]


# DRAM bytes per query of k_normals (k=16, float32) from one ncu capture each
# (dram__bytes_read.sum + dram__bytes_write.sum of a launch over its
# queries) on an 8M-point scene: tree-order queries and scattered serving
# queries.  A scaling constant: the full-size launches are too large to
# capture, and the traffic of a launch grows with the queries it answers,
# so the reported traffic is this figure times the queries of a launch.
TRAFFIC_PER_QUERY = {"tree_order": 126.8, "scattered": 160.5,
                     # the fused kNN + normal launch (k_normals with kNN outputs) on a
                     # 256-cloud ragged batch of 11.5M points, every point in tree order
                     "fused_tree_order": 102.1}


def roofline(ctx, stage_name, queries, traffic_kind, bytes_per_query=BYTES_PER_QUERY):
    """traffic_kind None: no ncu traffic figure for this kernel's launch."""
    peak, peak_kind = load_peaks()
    t_ms, cnt = ctx.stage(stage_name)
    if not cnt or t_ms <= 0:
        return None
    per_launch_ms = t_ms / cnt
    bytes_per_launch = bytes_per_query * queries / cnt
    achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
    traffic = TRAFFIC_PER_QUERY[traffic_kind] * queries / cnt if traffic_kind else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": "k_normals", "peak_kind": f"{peak_kind} hbm_gbs",
            "ms_per_launch": per_launch_ms, "bytes_per_launch": bytes_per_launch,
            "traffic_source": f"ncu bytes/query ({traffic_kind}) x queries" if traffic_kind else None}


BUILD_STAGES = ("build", "build.prep", "build.attempt", "build.levels", "build.subtree", "build.finish",
                "build.tnodes", "order", "normals")


def run_plain_workload(args, ctx):
    torch, N = ctx.torch, ctx.N
    from pptk_b200 import estimate_normals, synth
    pts = synth.lidar_scene(args.points, seed=2)
    n = len(pts)
    dev = torch.from_numpy(pts).cuda()
    evecs = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def step():
        N.call("pptkg_estimate_normals", N.ptr(dev), n, 0, N.MEM_DEVICE, args.k, ctypes.c_float(np.inf), None, n,
               1, N.PREC_AUTO, N.ptr(evecs), None, None, sp)

    for _ in range(args.warmup):
        step()
    ctx.lib.pptkg_profile_enable(1)
    ms, launches, clk = device_timed(ctx, step, args.steps)
    stages = {}
    for nm in BUILD_STAGES:
        t_, c_ = ctx.stage(nm)
        stages[nm] = t_ / max(c_, 1) if c_ else 0.0
    roof = roofline(ctx, "normals", n * args.steps, "tree_order")
    ctx.lib.pptkg_profile_enable(0)
    ms_max = ctx.max_over_ranks(ms)
    value = ctx.throughput(n, ms / 1e3)
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(pts).pin_memory().numpy()
        for _ in range(2):
            estimate_normals(host, args.k, np.inf, verbose=False)
        ctx.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = estimate_normals(host, args.k, np.inf, verbose=False)
        torch.cuda.synchronize()
        dt = ctx.max_over_ranks((time.perf_counter() - t0) / args.steps)
        e2e = {"value": ctx.world * n / dt, "unit": "queries/s", "h2d_bytes_per_step": int(pts.nbytes),
               "d2h_bytes_per_step": int(out.nbytes)}
    cpu = cpu_baseline_obj(pts, args) if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline else None
    return {"value": value, "ms_per_step": ms_max,
            "config": {"workload": f"lidar_scene_{n}_f32 estimate_normals k={args.k} r=inf, all points as queries "
                                   "(one drop-in call: device build + fused kNN+PCA)",
                       "points": n, "k": args.k, "l2": "inputs (240 MB) larger than L2 (126 MB); no flush",
                       "parallelism": f"replicas x{ctx.world}"},
            "e2e": e2e, "gpu_launches": launches, "stages_ms": stages, "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk}


def run_ragged_workload(args, ctx):
    """Ragged batch: 4,096 clouds (synth.ragged_clouds, seed 4, sizes
    log-uniform in [1k, 200k]); one step builds every cloud's tree in one
    forest build and answers kNN k=16 and normals k=16 for every point of
    every cloud -- one Forest.knn_normals traversal per point (the same
    results as Forest.knn + Forest.normals, which are timed beside it).
    Bucket size, lane_span, warm_bound, topk_min and warm_mult are picked by
    the autotuner on the first 256 clouds before timing."""
    torch = ctx.torch
    from pptk_b200 import autotune, ragged, synth
    k = args.k
    nc = args.clouds
    P, off = synth.ragged_clouds(nc, seed=4)
    n = len(P)
    dev = torch.from_numpy(P).cuda()
    if args.no_autotune:
        tuned = {"bucket": 64, "lane_span": None, "table": [], "knob_table": []}
    else:
        ns = min(256, nc)
        fs = ragged.Forest(dev[:int(off[ns])], off[:ns + 1])
        tuned = autotune.tune(lambda: fs.knn_normals(k), fs.set_bucket)
        del fs

    def step():
        f = ragged.Forest(dev, off)
        f.set_bucket(tuned["bucket"])
        f.knn_normals(k)

    def step_separate():
        f = ragged.Forest(dev, off)
        f.set_bucket(tuned["bucket"])
        f.knn(k)
        f.normals(k)

    for _ in range(args.warmup):
        step()
    ctx.lib.pptkg_profile_enable(1)
    ms, launches, clk = device_timed(ctx, step, args.steps)
    stages = {}
    for nm in BUILD_STAGES[:7] + ("forest.knn_normals",):
        t_, c_ = ctx.stage(nm)
        stages[nm] = {"ms_per_step": t_ / args.steps, "calls_per_step": c_ / args.steps}
    roof = roofline(ctx, "forest.knn_normals", n * args.steps, "fused_tree_order", BYTES_PER_QUERY_FUSED)
    ctx.lib.pptkg_profile_enable(0)
    ms_max = ctx.max_over_ranks(ms)
    value = ctx.throughput(n, ms / 1e3)
    # the same step as two calls (Forest.knn, then Forest.normals)
    step_separate()
    ctx.lib.pptkg_profile_enable(1)
    ms_sep, _, _ = device_timed(ctx, step_separate, args.steps)
    for nm in ("forest.knn", "forest.normals"):
        t_, c_ = ctx.stage(nm)
        stages[nm + " (separate calls)"] = {"ms_per_step": t_ / args.steps, "calls_per_step": c_ / args.steps}
    ctx.lib.pptkg_profile_enable(0)
    f = ragged.Forest(dev, off)
    f.set_bucket(tuned["bucket"])
    # the whole step (forest rebuild from the points + kNN + normals)
    # replayed from one CUDA graph; its results are checked against the
    # direct calls once
    buf = dev.clone()
    l0 = ctx.lib.pptkg_launch_count()
    cap_p, outs = f.capture_pipeline(buf, k)
    kernels_p = (ctx.lib.pptkg_launch_count() - l0) // 2  # one direct pass, one captured
    for _ in range(args.warmup):  # (the first launches upload the graph and map its memory)
        cap_p.replay()
    ms_p, _, _ = device_timed(ctx, cap_p.replay, args.steps)
    cap_p.check()
    ref_i, ref_c = f.knn(k)
    pipeline_ok = bool(torch.equal(outs["indices"], ref_i) and torch.equal(outs["counts"], ref_c)
                       and torch.equal(torch.nan_to_num(outs["normals"], nan=-9.0),
                                       torch.nan_to_num(f.normals(k), nan=-9.0)))
    del cap_p, outs, ref_i, ref_c
    # the same comparison on a small batch (512 clouds of 500-5,000
    # points), where launches and host round trips weigh more
    Ps, offs = synth.ragged_clouds(512, lo=500, hi=5000, seed=7)
    devs = torch.from_numpy(Ps).cuda()

    def step_small():
        fsm = ragged.Forest(devs, offs)
        fsm.set_bucket(tuned["bucket"])
        fsm.knn_normals(k)

    for _ in range(args.warmup):
        step_small()
    ms_sd, _, _ = device_timed(ctx, step_small, max(args.steps, 10))
    fsm = ragged.Forest(devs, offs)
    fsm.set_bucket(tuned["bucket"])
    bufs = devs.clone()
    cap_s, outs_s = fsm.capture_pipeline(bufs, k)
    for _ in range(args.warmup):
        cap_s.replay()
    ms_sg, _, _ = device_timed(ctx, cap_s.replay, max(args.steps, 10))
    cap_s.check()
    ri, rc = fsm.knn(k)
    small_ok = bool(torch.equal(outs_s["indices"], ri) and torch.equal(outs_s["counts"], rc))
    del cap_s, outs_s, fsm, bufs, devs
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(P).pin_memory().numpy()
        ctx.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fh = ragged.Forest(host, off)
            fh.set_bucket(tuned["bucket"])
            i, c, nn = fh.knn_normals(k)
        dt = ctx.max_over_ranks((time.perf_counter() - t0) / args.steps)
        e2e = {"value": ctx.world * n / dt, "unit": "queries/s", "h2d_bytes_per_step": int(P.nbytes),
               "d2h_bytes_per_step": int(i.nbytes + c.nbytes + nn.nbytes)}
    return {"value": value, "ms_per_step": ms_max,
            "config": {"workload": f"ragged batch of {nc} float32 clouds ({n} points, sizes log-uniform in "
                                   f"[1k, 200k]): forest build + kNN k={k} + normals k={k} for every point",
                       "clouds": nc, "points": n, "k": k, "l2": f"inputs ({P.nbytes / 1e9:.2f} GB) larger than L2",
                       "parallelism": f"replicas x{ctx.world}"},
            "autotune": {"bucket": tuned["bucket"], "lane_span": tuned["lane_span"],
                         "warm_bound": tuned.get("warm_bound"), "topk_min": tuned.get("topk_min"),
                         "warm_mult": tuned.get("warm_mult"),
                         "sample": "first 256 clouds", "table": tuned["table"],
                         "knob_table": tuned.get("knob_table")},
            "separate_calls": {"ms_per_step": ms_sep, "what": "the same step with Forest.knn and Forest.normals "
                                                             "as two traversals"},
            "graph_pipeline": {"value": ctx.world * n / (ctx.max_over_ranks(ms_p) / 1e3), "unit": "points/s",
                               "ms_per_step": ms_p, "direct_ms_per_step": ms_max, "equal_to_direct": pipeline_ok,
                               "kernels_in_graph": kernels_p,
                               "small_batch": {"clouds": 512, "points": int(len(Ps)), "ms_per_step": ms_sg,
                                               "direct_ms_per_step": ms_sd, "equal_to_direct": small_ok},
                               "what": "the whole step (forest rebuild + one kNN + normals traversal) replayed from one CUDA "
                                       "graph on a capture-ready forest"},
            "e2e": e2e, "gpu_launches": launches, "stages_ms": stages, "roofline": roof,
            "cpu_baseline": None, "clocks": clk}


def _scene_to_file(args):
    """Worker: writes one lidar scene (n points, seed) to path as .npy."""
    n, seed, path = args
    sys.path.insert(0, ROOT)
    from pptk_b200 import synth
    np.save(path, synth.lidar_scene(n, seed=seed))
    return path


def run_multitree_workload(args, ctx):
    """Serving over 64 resident trees (lidar scenes, seeds 100-163, sizes
    uniform in [1M, 10M]): Poisson arrivals of kNN (k uniform in 8..64),
    r-near (r uniform in [0.1, 1.0] m) and normal (k=16) requests with query
    batches log-uniform in [1k, 1M] points, plus 5% build requests of new
    clouds (0.5M-5M points); HBM admission budget 150 GB.  Measures the
    sustained throughput at saturation (a burst of the whole request list),
    then throughput and p50/p99 latency at fixed offered loads of a quarter
    (`latency`) and half (`latency_at_half_load`) of it."""
    import concurrent.futures as cf
    import multiprocessing as mpc
    import tempfile
    torch = ctx.torch
    from pptk_b200 import serving
    rng = np.random.default_rng(7)
    sizes = rng.integers(1_000_000, 10_000_001, 64)
    extra = rng.integers(500_000, 5_000_001, 4)
    tmp = tempfile.mkdtemp(prefix="pptk_b200_trees_")
    jobs = [(int(sz), 100 + i, os.path.join(tmp, f"t{i}.npy")) for i, sz in enumerate(sizes)]
    jobs += [(int(sz), 200 + i, os.path.join(tmp, f"b{i}.npy")) for i, sz in enumerate(extra)]
    with cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 4), mp_context=mpc.get_context("spawn")) as ex:
        paths = list(ex.map(_scene_to_file, jobs))
    clouds = [torch.from_numpy(np.load(p_)).cuda() for p_ in paths[:64]]
    new_clouds = [torch.from_numpy(np.load(p_)).cuda() for p_ in paths[64:]]
    for p_ in paths:
        os.remove(p_)
    os.rmdir(tmp)
    n_total = int(sizes.sum())
    srv = serving.Server(budget_bytes=150e9, slots=args.slots, max_batch_queries=args.max_batch)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids = [f.result() for f in [srv.build(c) for c in clouds]]
    build_s = time.perf_counter() - t0

    def make_requests(count, seed):
        r = np.random.default_rng(seed)
        out = []
        for _ in range(count):
            u = r.random()
            g = int(r.integers(0, 64))
            m = int(np.exp(r.uniform(np.log(1e3), np.log(1e6))))
            rows = torch.from_numpy(r.integers(0, len(clouds[g]), m)).cuda()
            if u < 0.05:
                out.append(("build", int(r.integers(0, len(new_clouds))), None))
            elif u < 0.45:
                out.append(("knn", g, (clouds[g][rows].contiguous(), int(r.integers(8, 65)))))
            elif u < 0.60:
                # r-near batches are capped at 4k points: about a tenth of
                # the points lie within ~1 m of the sensor, where a 1 m ball
                # holds ~1e5 points
                out.append(("rnear", g, (clouds[g][rows[:4000]].contiguous(), float(r.uniform(0.1, 1.0)))))
            else:
                out.append(("normals", g, rows.to(torch.int32)))
        return out

    def submit(req):
        kind, g, a = req
        if kind == "build":
            return srv.build(new_clouds[g])
        if kind == "knn":
            return srv.knn(ids[g], a[0], k=a[1])
        if kind == "rnear":
            return srv.rnear(ids[g], a[0], a[1])
        return srv.normals(ids[g], a, k=16)

    def queries(req):
        kind, g, a = req
        return 0 if kind == "build" else (len(a[0]) if kind in ("knn", "rnear") else len(a))

    built = []

    def finish(req, fut):
        res = fut.result()
        if req[0] == "build":
            built.append(res)

    def drop_built():
        while built:
            srv.drop(built.pop())

    def run_all(reqs):
        futs = [submit(rq) for rq in reqs]
        for i, rq in enumerate(reqs):
            finish(rq, futs[i])
            futs[i] = None  # drop the result

    run_all(make_requests(40, 1))
    drop_built()
    burst = make_requests(300, 2)
    q_burst = sum(queries(r_) for r_ in burst)
    clk_s = ClockSampler(ctx.local)
    clk_s.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run_all(burst)
    torch.cuda.synchronize()
    sat_s = time.perf_counter() - t0
    drop_built()
    sat = q_burst / sat_s
    # fixed offered loads (a quarter and half of the saturation rate),
    # Poisson arrivals of the same seeded request stream
    stream_reqs = make_requests(1500, 3)
    mean_q = np.mean([queries(r_) for r_ in stream_reqs])
    loads = {}
    for frac in (0.25, 0.5):
        rate = frac * sat / mean_q
        arr = np.random.default_rng(4)
        t_start = time.perf_counter()
        nxt = t_start
        pending = []
        sink = ResultSink(lambda rq, res: built.append(res) if rq[0] == "build" else None)
        for rq in stream_reqs:
            while time.perf_counter() < nxt:
                time.sleep(max(0.0, min(nxt - time.perf_counter(), 0.002)))
            sink.add(submit(rq), rq)
            pending.append((rq, None))
            nxt += arr.exponential(1.0 / rate)
            if time.perf_counter() - t_start > args.latency_seconds:
                break
        sink.wait()
        span = time.perf_counter() - t_start
        drop_built()
        st = srv.stats(since=t_start)
        with srv._cv:
            lat = [d[3] - d[2] for d in srv._done if d[2] >= t_start and d[0] != "build"]
        q_done = sum(queries(rq) for rq, _ in pending)
        loads[frac] = {"offered_queries_per_s": frac * sat, "achieved_queries_per_s": q_done / span,
                       "arrivals": "poisson", "requests": len(pending), "serving": percentiles(lat),
                       "by_kind": {kk: {"p50_ms": v["p50_s"] * 1e3, "p99_ms": v["p99_s"] * 1e3,
                                        "requests": v["requests"]}
                                   for kk, v in st.items() if isinstance(v, dict)}}
    clk = clk_s.stop()
    srv.close()
    value = ctx.throughput(q_burst, sat_s)
    return {"value": value, "ms_per_step": 1e3 * sat_s,
            "config": {"workload": f"serving over 64 resident lidar trees ({n_total} points, 1M-10M each): "
                                   "kNN k 8-64 / r-near r 0.1-1.0 m / normals k=16 requests, batches log-uniform "
                                   "1k-1M (r-near capped at 4k queries), 5% builds of 0.5M-5M clouds, budget 150 GB",
                       "trees": 64, "points": n_total, "burst_requests": len(burst), "slots": args.slots,
                       "parallelism": f"replicas x{ctx.world}"},
            "steps_note": "one step = a burst of 300 requests answered at saturation",
            "build": {"trees": 64, "points_per_s": n_total / build_s, "seconds": build_s},
            "latency": loads[0.25], "latency_at_half_load": loads[0.5],
            "e2e": None, "gpu_launches": None, "roofline": None, "cpu_baseline": None, "clocks": clk}


def run_scene_workload(args, ctx):
    """The 20M-point scene's other queries (config 2): kNN k=32 for every
    point (self queries, tree order), r-near r=0.5 m hit counts for every
    point, and the r-near hit lists for 20k random points (filling them for
    every point is not feasible on any machine: a point within ~1 m of the
    sensor has ~1e5 hits at r=0.5 m, about a tenth of the points lie there).
    `value` is the kNN k=32 rate; the r-near figures sit beside it."""
    torch, N = ctx.torch, ctx.N
    from pptk_b200 import kdtree, synth
    pts = synth.lidar_scene(args.points, seed=2)
    n = len(pts)
    dev = torch.from_numpy(pts).cuda()
    tree = kdtree._build(dev)
    k = 32
    idx = torch.empty((n, k), dtype=torch.int32, device="cuda")
    cnt = torch.empty((n,), dtype=torch.int32, device="cuda")
    sp = N.torch_stream()

    def knn_step():
        N.call("pptkg_knn_self", tree._h, None, n, N.MEM_DEVICE, k, float("inf"), N.ptr(idx), N.ptr(cnt), sp)

    for _ in range(args.warmup):
        knn_step()
    ctx.lib.pptkg_profile_enable(1)
    ms, launches, clk = device_timed(ctx, knn_step, args.steps)
    ctx.lib.pptkg_profile_enable(0)
    ms_max = ctx.max_over_ranks(ms)
    value = ctx.throughput(n, ms / 1e3)
    # r-near counts for every point (the count pass of count / scan / fill)
    r = 0.5
    off = torch.empty((n + 1,), dtype=torch.int64, device="cuda")
    total = ctypes.c_int64()

    def count_step():
        N.call("pptkg_rnear_count", tree._h, None, None, n, 0, N.MEM_DEVICE, r, N.ptr(off), ctypes.byref(total), sp)

    count_step()
    ms_c, _, _ = device_timed(ctx, count_step, args.steps)
    hits = int(total.value)
    # hit lists for a sample
    rows = torch.from_numpy(np.random.default_rng(13).integers(0, n, 20_000).astype(np.int32)).cuda()
    q = dev[rows.long()].contiguous()

    def sample_step():
        return kdtree.rnear(tree, q, r)

    sample_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o_, h_ = sample_step()
    torch.cuda.synchronize()
    ms_s = (time.perf_counter() - t0) / args.steps * 1e3
    sample_hits = int(o_[-1].item())
    cpu = None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        sel = np.sort(np.random.default_rng(0).choice(n, size=1_000_000, replace=False))
        ref = O.RefTree(np.ascontiguousarray(pts[sel])) if O.ref_available() else O.PortTree(
            np.ascontiguousarray(pts[sel]))
        t0 = time.perf_counter()
        ref.knn_self(np.arange(len(sel), dtype=np.int32), k, nthreads=0)
        dt = time.perf_counter() - t0
        cpu = {"value": len(sel) / dt, "unit": "queries/s", "cores": O.ref_lib().ref_max_threads(),
               "kind": "reference" if O.ref_available() else "port",
               "sample": f"kNN k={k} self queries over a 1M-point random sample of the scene (tree built beforehand, "
                         f"{dt:.1f} s)"}
    return {"value": value, "ms_per_step": ms_max,
            "config": {"workload": f"lidar_scene_{n}_f32: kNN k={k} self queries for every point (tree order)",
                       "points": n, "k": k, "parallelism": f"replicas x{ctx.world}"},
            "rnear": {"r": r, "count_all_points_ms": ms_c, "count_queries_per_s": n / (ms_c / 1e3),
                      "total_hits_all_points": hits,
                      "sample_queries": 20_000, "sample_hits": sample_hits, "sample_count_and_fill_ms": ms_s,
                      "note": "hit lists for all points would be "
                              f"{hits * 4 / 1e9:.0f} GB; filled for a 20k-point sample only"},
            "e2e": None, "gpu_launches": launches, "roofline": None, "cpu_baseline": cpu, "clocks": clk}


def percentiles(lat_s):
    a = np.asarray(lat_s, dtype=np.float64) * 1e3
    return {"p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)), "requests": int(a.size)}


def run_serving_workload(args, ctx):
    torch = ctx.torch
    from pptk_b200 import estimate_normals, kdtree, serving, synth
    pts = synth.lidar_scene(args.points, seed=2)
    n = len(pts)
    k = args.k
    dev = torch.from_numpy(pts).cuda()
    warm_mix = synth.request_mix(n, n, seed=10)
    mix = synth.request_mix(n, n, seed=11)
    per_step = sum(len(r) for _, r in mix)
    n_norm = sum(len(r) for kind, r in mix if kind == "normals")
    n_knn = per_step - n_norm

    def device_requests(m):
        out = []
        for kind, rows in m:
            r = torch.from_numpy(rows).cuda()
            out.append((kind, dev[r.long()].contiguous() if kind == "knn" else r))
        return out

    warm_dev, mix_dev = device_requests(warm_mix), device_requests(mix)
    srv = serving.Server(budget_bytes=150e9, slots=args.slots, max_batch_queries=args.max_batch,
                         max_host_batch_queries=args.max_host_batch, batch_ms=args.batch_ms)
    tid = srv.build(dev).result()

    def submit(reqs):
        return [srv.knn(tid, a, k=k) if kind == "knn" else srv.normals(tid, a, k=k) for kind, a in reqs]

    def serve(reqs):
        for f in submit(reqs):
            f.result()

    for _ in range(args.warmup):
        serve(warm_dev)
    ctx.lib.pptkg_profile_enable(1)
    ms, launches, clk = device_timed(ctx, lambda: serve(mix_dev), args.steps)
    stages = {}
    for nm in ("multi.knn", "multi.normals", "normals.refine64", "order"):
        t_, c_ = ctx.stage(nm)
        stages[nm] = {"ms_total_per_step": t_ / args.steps, "launches_per_step": c_ / args.steps}
    roof = roofline(ctx, "multi.normals", n_norm * args.steps, "scattered")
    ctx.lib.pptkg_profile_enable(0)
    ms_max = ctx.max_over_ranks(ms)
    value = ctx.throughput(per_step, ms / 1e3)

    # latency at fixed offered loads: Poisson arrivals at half (`latency`)
    # and a quarter (`latency_at_quarter_load`) of the measured serving
    # throughput, requests drawn in stream order
    def poisson_latency(frac, seed):
        rng = np.random.default_rng(seed)
        offered = frac * per_step / (ms_max / 1e3)
        mean_m = per_step / len(mix_dev)
        t_start = time.perf_counter()
        sink, i = ResultSink(), 0
        next_t = t_start
        while time.perf_counter() - t_start < args.latency_seconds:
            now = time.perf_counter()
            if now < next_t:
                time.sleep(min(next_t - now, 0.002))
                continue
            kind, a = mix_dev[i % len(mix_dev)]
            sink.add(srv.knn(tid, a, k=k) if kind == "knn" else srv.normals(tid, a, k=k))
            i += 1
            next_t += rng.exponential(mean_m / offered)
        sink.wait()
        st = srv.stats(since=t_start)
        with srv._cv:
            lat_all = [d[3] - d[2] for d in srv._done if d[2] >= t_start and d[0] in ("knn", "normals")]
        return {"offered_queries_per_s": offered, "arrivals": "poisson",
                "serving": percentiles(lat_all),
                "serving_by_kind": {kk: {"p50_ms": v["p50_s"] * 1e3, "p99_ms": v["p99_s"] * 1e3,
                                         "requests": v["requests"]}
                                    for kk, v in st.items() if isinstance(v, dict)}}

    latency = poisson_latency(0.5, 12)
    latency_q = poisson_latency(0.25, 13)

    # plain per-call drop-in on a bounded sample of the same stream
    tree = kdtree._build(dev)
    sample = mix[:args.plain_sample]

    def plain_calls(reqs, host, scene):
        lat, q = [], 0
        for kind, rows in reqs:
            if host:
                a = scene[rows] if kind == "knn" else rows
            else:
                r = torch.from_numpy(rows).cuda()
                a = dev[r.long()].contiguous() if kind == "knn" else r
                torch.cuda.synchronize()
            t0 = time.perf_counter()
            if kind == "knn":
                res = kdtree.knn(tree, a, k)
            else:
                res = estimate_normals(scene if host else dev, k, np.inf, subsample=a, verbose=False)
            torch.cuda.synchronize()
            lat.append(time.perf_counter() - t0)
            q += len(rows)
            del res
        return q / sum(lat), lat

    # warm-up: the largest request of each kind, so the device memory pool
    # has grown to the sample's needs before the timed calls
    warm = [max((r for r in sample if r[0] == kd), key=lambda r: len(r[1])) for kd in ("knn", "normals")]
    plain_calls(warm, False, pts)
    plain_qps, plain_lat = plain_calls(sample, False, pts)
    plain = {"value": plain_qps, "unit": "queries/s", "latency": percentiles(plain_lat),
             "sample": f"first {len(sample)} requests of the stream ({sum(len(r) for _, r in sample)} queries), "
                       "one call each, device inputs"}
    if not args.no_e2e:
        host_pts = torch.from_numpy(pts).pin_memory().numpy()
        plain_calls(warm, True, host_pts)
        h_qps, h_lat = plain_calls(sample, True, host_pts)
        plain["e2e"] = {"value": h_qps, "unit": "queries/s", "latency": percentiles(h_lat),
                        "inputs": "host numpy (pinned scene); results returned as numpy"}
    del tree

    # serving e2e: pinned host inputs, numpy results
    e2e = None
    if not args.no_e2e:
        host_reqs = []
        h2d = d2h = 0
        for kind, rows in mix:
            a = torch.from_numpy(pts[rows] if kind == "knn" else rows).pin_memory().numpy()
            host_reqs.append((kind, a))
            h2d += a.nbytes
            d2h += len(rows) * (4 * k + 4 if kind == "knn" else 12)
        serve(host_reqs)
        ctx.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            serve(host_reqs)
        torch.cuda.synchronize()
        dt = ctx.max_over_ranks((time.perf_counter() - t0) / args.steps)
        e2e = {"value": ctx.world * per_step / dt, "unit": "queries/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h)}
    srv.close()
    cpu = (serving_cpu_baseline(pts, mix, args)
           if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline else None)
    return {"value": value, "ms_per_step": ms_max,
            "config": {"workload": f"lidar scene {n} f32, resident tree, server; {len(mix)} requests/step: "
                                   f"{n_knn} kNN k={k} + {n_norm} normal k={k} queries",
                       "points": n, "k": k, "queries_per_step": per_step, "slots": args.slots,
                       "batch_ms": args.batch_ms, "l2": "inputs > L2, no flush", "unit": "request row",
                       "parallelism": f"replicas x{ctx.world}"},
            "plain": plain, "latency": latency, "latency_at_quarter_load": latency_q,
            "e2e": e2e, "gpu_launches": launches, "stages_ms": stages, "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk}


def angle_stats(a, b):
    """p50/p99/max of the unsigned angle (rad) between row vectors of two
    CUDA tensors, over rows finite in both."""
    import torch
    a = a.double()
    b = b.double()
    ok = torch.isfinite(a).all(1) & torch.isfinite(b).all(1)
    a, b = a[ok], b[ok]
    cr = torch.linalg.norm(torch.cross(a, b, dim=1), dim=1)
    dt = (a * b).sum(1).abs()
    ang = torch.sort(torch.atan2(cr, dt)).values
    n = ang.numel()
    if n == 0:
        return {"p50": None, "p99": None, "max": None, "rows": 0}
    return {"p50": float(ang[int(0.5 * (n - 1))]), "p99": float(ang[int(0.99 * (n - 1))]), "max": float(ang[-1]),
            "rows": int(n)}


def precision_report():
    """FP32 normal path against FP64 on the configs' clouds: every row
    against the device FP64 path, and a sample of rows against the CPU FP64
    oracle (float64 covariance of the same neighbours, numpy eigh)."""
    import torch
    from oracle import oracle as O
    from pptk_b200 import estimate_normals, synth
    out = {}
    cases = [("uniform_200k_f32_k16", lambda: synth.uniform_cube(200_000, seed=0), 16, "auto"),
             ("lidar_scene_20M_f32_k16", lambda: synth.lidar_scene(20_000_000, seed=2), 16, "auto"),
             ("planar_patches_10M_f64_k24", lambda: synth.planar_patches(10_000_000, seed=3)[0], 24, "fp32")]
    for name, gen, k, prec in cases:
        P = gen()
        dev = torch.from_numpy(P).cuda()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n32 = estimate_normals(dev, k, np.inf, precision=prec, verbose=False)
        torch.cuda.synchronize()
        t32 = time.perf_counter() - t0
        n64 = estimate_normals(dev, k, np.inf, precision="fp64", verbose=False)
        rows = np.sort(np.random.default_rng(5).choice(len(P), size=min(20_000, len(P)), replace=False)).astype(
            np.int32)
        _, _, _, nb = O.port_estimate_normals(P, k, np.inf, subsample=rows, num_eigen=3, want_nbrs=True)
        w, V, _ = O.normals_fp64(P, nb)
        ref = torch.from_numpy(np.ascontiguousarray(V[:, 0, :])).cuda()
        out[name] = {"dtype": str(P.dtype), "k": k, "fp32_path": prec,
                     "fp32_path_queries_per_s": len(P) / t32,
                     "vs_device_fp64_all_rows": angle_stats(n32, n64),
                     "vs_cpu_fp64_oracle_sample": angle_stats(n32[torch.from_numpy(rows).cuda().long()], ref),
                     "device_fp64_vs_cpu_fp64_oracle_sample": angle_stats(
                         n64[torch.from_numpy(rows).cuda().long()], ref)}
        del dev, n32, n64
    return out


WORKLOADS = {"serving": run_serving_workload, "plain": run_plain_workload, "ragged": run_ragged_workload,
             "multitree": run_multitree_workload, "scene": run_scene_workload}

# keys of a workload's result that go to the detail lines (bulky, not headline figures)
DETAIL_KEYS = ("stages_ms", "autotune", "precision", "rnear", "build", "steps_note")


def _lat(d):
    """p50/p99 of a latency block, compact."""
    if not d:
        return None
    s = d.get("serving", d)
    return {"offered_queries_per_s": d.get("offered_queries_per_s"), "p50_ms": s.get("p50_ms"),
            "p99_ms": s.get("p99_ms"), "requests": s.get("requests")}


def _precision_summary(prec):
    """p99 / max angular error (rad) of the FP32 path against the CPU FP64
    oracle on 20k sampled rows, per cloud."""
    return {name: [v["vs_cpu_fp64_oracle_sample"]["p99"], v["vs_cpu_fp64_oracle_sample"]["max"]]
            for name, v in prec.items()}


def compact_serving(res):
    """The headline figures of the serving workload, in a few hundred bytes."""
    plain = res.get("plain") or {}
    out = {"plain": {"value": plain.get("value"), "unit": "queries/s",
                     "p50_ms": (plain.get("latency") or {}).get("p50_ms"),
                     "p99_ms": (plain.get("latency") or {}).get("p99_ms"),
                     "e2e_value": (plain.get("e2e") or {}).get("value")},
           "latency": _lat(res.get("latency")), "latency_at_quarter_load": _lat(res.get("latency_at_quarter_load"))}
    if plain.get("value"):
        out["serving_over_plain"] = res["value"] / plain["value"]
    return out


def run_config(name, args, ctx):
    """One other configuration, briefly (3 warm-up, <= 5 timed steps), as a
    compact summary plus its full result for the detail lines."""
    a = argparse.Namespace(**vars(args))
    a.steps, a.warmup = max(1, min(args.steps, 5)), 3
    a.no_cpu_baseline, a.no_e2e, a.latency_seconds = True, True, 2.0
    if name == "ragged":
        a.no_e2e = False
    res = WORKLOADS[name](a, ctx)
    summary = {"value": res["value"], "unit": "queries/s" if name != "ragged" else "points/s",
               "ms_per_step": res["ms_per_step"]}
    if name == "scene":
        rn = res["rnear"]
        summary["rnear_r0.5"] = {"count_all_ms": rn["count_all_points_ms"], "hits": rn["total_hits_all_points"],
                                 "fill_20k_ms": rn["sample_count_and_fill_ms"]}
    elif name == "ragged":
        st = res["stages_ms"]
        summary["stage_ms"] = {k: round(v["ms_per_step"], 1) for k, v in st.items()
                               if k in ("build", "forest.knn_normals")}
        summary["separate_calls_ms"] = round(res["separate_calls"]["ms_per_step"], 1)
        gp = res["graph_pipeline"]
        summary["graph_step_ms"] = round(gp["ms_per_step"], 1)
        summary["graph_step_equal"] = gp["equal_to_direct"]
        summary["graph_vs_direct_small_ms"] = [round(gp["small_batch"]["ms_per_step"], 2),
                                               round(gp["small_batch"]["direct_ms_per_step"], 2)]
        summary["e2e_value"] = (res["e2e"] or {}).get("value")
    elif name == "multitree":
        lq, lh = _lat(res["latency"]), _lat(res["latency_at_half_load"])
        summary["p50_p99_ms_quarter_load"] = [round(lq["p50_ms"], 1), round(lq["p99_ms"], 1)]
        summary["p50_p99_ms_half_load"] = [round(lh["p50_ms"], 1), round(lh["p99_ms"], 1)]
        summary["build_points_per_s"] = res["build"]["points_per_s"]
    clk = res.get("clocks") or {}
    summary["sm_mhz"] = clk.get("sm_mhz")
    if clk.get("reasons"):
        summary["clock_reasons"] = clk.get("reasons")
    return summary, res


def _round(x, digits=4):
    """Floats to `digits` significant digits, recursively (keeps the headline
    line short)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: _round(v, digits) for k, v in x.items()}
    if isinstance(x, list):
        return [_round(v, digits) for v in x]
    return x


def run_ours(args):
    ctx = Ctx()
    tuned = {}
    for kv in args.tune:
        name, val = kv.split("=", 1)
        ctx.N.tune_set(name, int(val))
        tuned[name] = int(val)
    ctx.lib.pptkg_profile_enable.argtypes = [ctypes.c_int]
    ctx.lib.pptkg_launch_count.restype = ctypes.c_int64
    res = WORKLOADS[args.workload](args, ctx)
    details = {}
    one = ctx.rank == 0 and ctx.world == 1
    if one and not args.no_precision:
        details["precision"] = precision_report()
    configs = {}
    if one and args.workload == "serving" and args.configs:
        for name in [c for c in args.configs.split(",") if c]:
            summary, full = run_config(name, args, ctx)
            configs[name] = summary
            details[f"config.{name}"] = full
    if ctx.rank == 0:
        for key in DETAIL_KEYS:
            if key in res:
                details[key] = res.pop(key)
        if args.workload == "serving":
            details["plain"] = res.get("plain")
            details["latency"] = {"half_load": res.get("latency"), "quarter_load": res.get("latency_at_quarter_load")}
            res.update(compact_serving(res))
        for name, d in details.items():
            print(json.dumps({"detail": name, "data": d}, default=str), flush=True)
        line = {"metric": METRIC, "value": res.pop("value"), "unit": "queries/s", "n_gpus": ctx.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res.pop("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic"}
        line.update(_round(res))
        if "precision" in details:
            line["precision_fp32_vs_fp64_oracle"] = _round(_precision_summary(details["precision"]), 3)
        if configs:
            line["configs"] = _round(configs)
        if tuned:
            line["config"]["tune"] = tuned
        print(json.dumps(line), flush=True)
    ctx.finish()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
