"""Benchmark of the pptk hot path on B200: kNN + PCA normal queries per second.

Workload (normals leg): a 20M-point float32 lidar-like
scene (pptk_b200.synth.lidar_scene, seed 2); one step is one drop-in
``estimate_normals(points, k=16, r=inf)`` call over all points -- the device
k-d tree build, the fused kNN (k=16, the point itself included) + covariance
+ eigensolve for every point, and the normals written out.

* ``value``: queries/s with the points already in HBM (C ABI, device
  pointers), CUDA events on the launching stream; the points (240 MB) are
  larger than L2, so no flush is needed between steps.
* ``e2e``: the same call through the public Python API with host numpy
  arrays (pinned), host<->device copies inside the timed region.
* ``roofline``: the fused kNN+PCA kernel's algorithmic bytes (216 B per
  query: the query point, 16 neighbour points, the normal) over its measured
  time, against the measured HBM copy bandwidth.
* ``cpu_baseline``: the reference's own k-d tree (compiled from its sources
  in oracle/_ref) with the restated normal loop, on a bounded sample, using
  every host core.

``--impl reference`` times only that CPU reference path on the same metric.
Multi-GPU (torchrun): every rank runs an independent replica of the
workload (weak scaling); there is no collective on the data path.
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


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--points", type=int, default=20_000_000)
    p.add_argument("--k", type=int, default=16)
    p.add_argument("--cpu-sample", type=int, default=1_000_000)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
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


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from pptk_b200 import synth
    pts = synth.lidar_scene(args.points, seed=2)
    vals = []
    for i in range(args.warmup + args.steps):
        qps, threads, dt, kind, n = cpu_reference(pts, args.k, args.cpu_sample, seed=i)
        if i >= args.warmup:
            vals.append((qps, dt))
    value = float(np.mean([v[0] for v in vals]))
    ms = float(np.mean([v[1] for v in vals])) * 1e3
    sample = (f"{n} points drawn without replacement from the {args.points}-point scene each step; tree build + "
              f"kNN k={args.k} + covariance + Jacobi eigensolve per point ({kind}; TBB absent: OpenMP over the "
              f"reference's per-query calls)")
    line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"lidar_scene_{args.points}_f32 estimate_normals k={args.k} r=inf (sampled)",
                       "points": args.points, "k": args.k},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from pptk_b200 import _native as N
    from pptk_b200 import estimate_normals, synth
    lib = N.lib()
    lib.pptkg_profile_enable.argtypes = [ctypes.c_int]
    lib.pptkg_profile_get.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int64)]
    lib.pptkg_launch_count.restype = ctypes.c_int64

    pts = synth.lidar_scene(args.points, seed=2)
    n = len(pts)
    dev = torch.from_numpy(pts).cuda()
    evecs = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step():
        N.call("pptkg_estimate_normals", N.ptr(dev), n, 0, N.MEM_DEVICE, args.k, ctypes.c_float(np.inf), None, n,
               1, N.PREC_AUTO, N.ptr(evecs), None, None, sp)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    lib.pptkg_profile_enable(1)
    l0 = lib.pptkg_launch_count()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = (lib.pptkg_launch_count() - l0) // max(args.steps, 1)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps

    def stage(name):
        t, c = ctypes.c_double(), ctypes.c_int64()
        lib.pptkg_profile_get(name.encode(), ctypes.byref(t), ctypes.byref(c))
        return t.value, c.value

    norm_ms, norm_cnt = stage("normals")
    build_ms, build_cnt = stage("build")
    stages = {}
    for nm in ("build", "build.prep", "build.attempt", "build.levels", "build.subtree", "build.finish",
               "build.tnodes", "order", "normals"):
        t_, c_ = stage(nm)
        stages[nm] = t_ / max(c_, 1) if c_ else 0.0
    lib.pptkg_profile_enable(0)
    ms_t = torch.tensor([ms], device="cuda")
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * n / (ms_max / 1e3)

    # e2e through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(pts).pin_memory().numpy()
        for _ in range(2):
            estimate_normals(host, args.k, np.inf, verbose=False)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = estimate_normals(host, args.k, np.inf, verbose=False)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.steps
        dt_t = torch.tensor([dt], device="cuda")
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(dt_t, op=dist.ReduceOp.MAX)
        e2e = {"value": world * n / float(dt_t.item()), "unit": "queries/s", "h2d_bytes_per_step": int(pts.nbytes),
               "d2h_bytes_per_step": int(out.nbytes)}

    peak, peak_kind = load_peaks()
    norm_launch_ms = norm_ms / max(norm_cnt, 1)
    achieved = BYTES_PER_QUERY * n / (norm_launch_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            qps, threads, dt, kind, ns = cpu_reference(pts, args.k, args.cpu_sample)
            cpu = {"value": qps, "unit": "queries/s", "cores": threads, "kind": kind,
                   "sample": f"{ns} random points of the scene: tree build + kNN k={args.k} + PCA per point "
                             f"({dt:.1f} s)"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "queries/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"lidar_scene_{n}_f32 estimate_normals k={args.k} r=inf, all points as "
                                       "queries (device build + fused kNN+PCA)",
                           "points": n, "k": args.k, "l2": "inputs (240 MB) larger than L2 (126 MB); no flush",
                           "parallelism": f"replicas x{world}"},
                "e2e": e2e,
                "gpu_launches": int(launches),
                "stages_ms": stages,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None,
                             "kernel": "k_normals (fused kNN+PCA)", "peak_kind": peak_kind},
                "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
