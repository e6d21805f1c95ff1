#!/usr/bin/env python
"""Benchmark of the STRATUM frame path on B200: shaded rays/s at 1600x900.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the plain single-view GPU frame at 1600x900, seed 0x5EED, six fixed
poses, 64-sample stationary accumulation): one step renders one shaded sample
of each of the six views -- stepCamera, lot refresh, hierarchy refresh, trace,
shade and resolve -- i.e. 6 x 1,440,000 shaded primary rays.  Inputs (lot
tables, 64 MiB hierarchies, frame buffers) are resident in HBM; L2 is flushed
between timed steps by a 256 MiB write that is outside the timed region.

`e2e` is the same metric through the one C-ABI call a user makes per view
(stratum_frame) with the step's input copied from pinned host memory and the
RGBA8 frame copied back, both inside the timed region.

Multi-GPU: views are independent, so N ranks run N replicas (weak scaling) with
no data-path collective; the reported time is the max over ranks.

`--impl reference` times the reference's own renderer (its kernels compiled as
host C++, oracle/_ref) on the host cores with every thread, on a bounded
sample of the same workload (a 48-row band of each pose per step).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
SEED = 0x5EED
WIDTH, HEIGHT = 1600, 900

# The six fixed poses of the 1600x900 workload.  `origin` is the 64-bit lot
# address (xl, xh, zl, zh) the camera position is relative to (before the
# floating-origin rebase).
POSES = {
    "street": {"origin": [0, 0, 0, 0], "pos": (17.0, 1.7, 0.0), "yaw": 0.0, "pitch": 0.0},
    "rooftop": {"origin": [0, 0, 0, 0], "pos": (17.0, 40.0, 0.0), "yaw": math.pi / 2, "pitch": 0.0},
    "aerial": {"origin": [0, 0, 0, 0], "pos": (0.0, 300.0, 0.0), "yaw": 0.6, "pitch": -math.pi / 6},
    "canal": {"origin": [28, 0, 1, 0], "pos": (0.0, 0.5, 0.0), "yaw": 0.0, "pitch": 0.0},
    "park": {"origin": [1, 0, 8, 0], "pos": (0.0, 2.0, -16.0), "yaw": 0.0, "pitch": 0.0},
    "avenue": {"origin": [0, 0, 0, 0], "pos": (17.99, 12.0, 0.0), "yaw": 0.0, "pitch": -2.0 * math.pi / 180},
}

# Algorithmic FP32 lane operations per shaded ray of each pose (whole path, and
# the trace kernel alone), from the reference algorithm: oracle/count_work.py
# weights each unit of work by its source-level FP32 operation count and
# multiplies by the instrumented oracle's counts at these poses (first sample,
# every 4th row of the 1600x900 frame).
OPS_PER_RAY = {  # pose: (whole path, trace only)
    "street": (14317.2, 13062.8),
    "rooftop": (9185.1, 8421.9),
    "aerial": (12696.3, 11808.9),
    "canal": (7583.5, 6626.1),
    "park": (10787.8, 9618.4),
    "avenue": (20391.0, 19066.5),
}
# DRAM bytes per traced ray of tracePrimary from an ncu capture of the street
# pose (profiles/tracePrimary_street_1600x900.md); None until captured.
TRACE_DRAM_BYTES_PER_RAY = None

METRIC = "shaded rays/s @1600x900"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-rows", type=int, default=48, help="rows per pose in a CPU sample")
    ap.add_argument("--poses", default=",".join(POSES), help="comma-separated subset of the six poses (profiling)")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="length of each serving run (0: skip)")
    ap.add_argument("--serve-views", type=int, default=8, help="views per serving batch")
    a = ap.parse_args(argv)
    a.poses = [p for p in a.poses.split(",") if p]
    unknown = set(a.poses) - set(POSES)
    if unknown:
        ap.error(f"unknown poses {sorted(unknown)}")
    return a


# ---------------------------------------------------------------- distributed
def dist_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_dist(world):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU legs
def cpu_lib():
    """The reference renderer built from its own sources (oracle/_ref), else the oracle port."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol
    if ol.ref_available():
        return ol, ol.RefLib(), "reference"
    return ol, ol.Oracle(), "port"


def cpu_sample(ol, lib, rows, steps=1, warmup=0):
    """Time trace + shade + resolve of a `rows`-row band at the middle of each
    pose's 1600x900 frame on all host threads.  Table set-up is untimed."""
    nthreads = os.cpu_count() or 1
    states = [ol.setup_pose(lib, SEED, p["pos"], p["yaw"], p["pitch"], WIDTH, HEIGHT, origin=p["origin"])
              for p in POSES.values()]
    P = WIDTH * HEIGHT
    bufs = [(np.zeros(P * 4, np.float32), np.zeros(P * 4, np.float32), np.zeros(P * 4, np.float32),
             np.zeros(P * 4, np.float32), np.zeros(P, np.uint32)) for _ in states]
    y0 = HEIGHT // 2 - rows // 2
    times = []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        for s, (hit, surf, lin, hist, px) in zip(states, bufs):
            lib.trace(s.World, s.Nodes, s.Origin, s.C, hit, surf, WIDTH, HEIGHT, row0=y0, rows=rows, nthreads=nthreads)
            lib.shade(s.World, s.Origin, s.C, hit, surf, lin, WIDTH, HEIGHT, row0=y0, rows=rows, nthreads=nthreads)
        for s, (hit, surf, lin, hist, px) in zip(states, bufs):
            lib.resolve_rows(lin, hist, px, s.C, hit, surf, WIDTH, HEIGHT, y0, rows, nthreads=nthreads)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
    rays = rows * WIDTH * len(states)
    return rays, times, nthreads


def reference_arm(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    ol, lib, kind = cpu_lib()
    rays, times, nthreads = cpu_sample(ol, lib, args.cpu_rows, steps=args.steps, warmup=args.warmup)
    total = sum(times)
    value = rays * len(times) / total
    sample = f"{args.cpu_rows}-row band at mid-frame of each of the 6 poses at 1600x900 ({rays} rays) per step"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural world, fixed poses)",
            "config": {"workload": "plain single-view frame 1600x900, seed 0x5EED, six poses", "width": WIDTH,
                       "height": HEIGHT, "poses": list(POSES), "device": "host CPU"},
            "cpu_baseline": {"value": value, "unit": "rays/s", "cores": nthreads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def issue_peak(torch, sb):
    """Measured FP32 lane-op rate of this GPU (stratum_issueProbe)."""
    out = torch.zeros(1, device="cuda")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8, 4096
    s = torch.cuda.current_stream()
    for _ in range(2):
        sb.call("stratum_issueProbe", sb.ptr(out), blocks, iters, s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(5):
        e0.record()
        sb.call("stratum_issueProbe", sb.ptr(out), blocks, iters, s.cuda_stream)
        e1.record()
        e1.synchronize()
        best = max(best, blocks * 256 * iters * 16 / (e0.elapsed_time(e1) * 1e-3))
    return best


def serve_poisson(rate, sessions, duration_s, widths, budget, max_views, streams, tune, seed=1):
    """Open-loop serving: Poisson arrivals at `rate` requests/s spread uniformly
    over `sessions` sessions for `duration_s` seconds.  Each session walks its
    camera through 64-bit lot space at a speed uniform in 1-50 m/s with a yaw
    drift uniform in +-10 deg/s; every request renders one new sample at the
    session's current pose.  A warm-up request per session (untimed) admits them
    all first.  Latency = submit -> frame back in host memory."""
    from stratum_hyperdetail_b200.server import Pose, Server
    rng = np.random.default_rng(seed)
    srv = Server(budget, max_views=max_views, streams=streams, tune=tune)
    cells = 36.0
    state = []
    for i in range(sessions):
        w = int(widths[rng.integers(len(widths))])
        h = int(round(w * 9 / 16))
        sid = srv.open(int(rng.integers(0, 2**31 - 1)), w, h)
        state.append({"sid": sid, "ox": int(rng.integers(0, 2**64, dtype=np.uint64)),
                      "oz": int(rng.integers(0, 2**64, dtype=np.uint64)), "x": float(rng.uniform(-18, 18)),
                      "z": float(rng.uniform(-18, 18)), "y": float(rng.uniform(1.5, 60.0)),
                      "yaw": float(rng.uniform(0, 2 * math.pi)), "pitch": float(rng.uniform(-0.25, 0.0)),
                      "speed": float(rng.uniform(1.0, 50.0)), "drift": math.radians(float(rng.uniform(-10, 10))),
                      "t": 0.0, "w": w, "h": h})

    def pose_at(s, t):
        dt = t - s["t"]
        s["t"] = t
        s["yaw"] += s["drift"] * dt
        s["x"] += math.sin(s["yaw"]) * s["speed"] * dt
        s["z"] += math.cos(s["yaw"]) * s["speed"] * dt
        for axis, o in (("x", "ox"), ("z", "oz")):  # keep the local position inside the cell
            c = math.floor((s[axis] + 18.0) / cells)
            s[o] = (s[o] + c) % 2**64
            s[axis] -= c * cells
        return Pose.make((s["ox"] & 0xFFFFFFFF, s["ox"] >> 32, s["oz"] & 0xFFFFFFFF, s["oz"] >> 32),
                         (s["x"], s["y"], s["z"]), s["yaw"], s["pitch"])

    warm = [srv.submit(s["sid"], pose_at(s, 0.0)) for s in state]
    for r in warm:
        srv.wait_status(r, 600000)
    base = srv.stats()
    times, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration_s:
            break
        times.append(t)
    who = rng.integers(0, sessions, len(times))
    rids, rays = [], 0
    t0 = time.perf_counter()
    for t, k in zip(times, who):
        lag = t - (time.perf_counter() - t0)
        if lag > 0:
            time.sleep(lag)
        s = state[int(k)]
        rids.append(srv.submit(s["sid"], pose_at(s, t)))
        rays += s["w"] * s["h"]
    lat = []
    for r in rids:
        info = srv.wait(r, 600000)
        if info.status == 0:
            lat.append(info.latency_ms)
    span = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat = np.array(lat) if lat else np.array([float("nan")])
    return {"requests": len(rids), "completed": int(len(lat)), "rate_offered": rate, "duration_s": duration_s,
            "sessions": sessions, "widths": list(widths), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "rays_per_s": rays / span, "batches": st["batches"] - base["batches"],
            "admissions": st["admissions"], "evictions": st["evictions"], "budget_gb": budget / 2**30,
            "resident_gb": st["resident_bytes"] / 2**30, "max_views": max_views, "streams": streams}


def timed_steps(torch, stream, steps, flush, body):
    """Run `steps` timed steps: L2 flush (untimed), then `body(events)` between
    two CUDA events on `stream`.  Returns per-step milliseconds and whatever
    `body` returns per step."""
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    ms, out = [], []
    for _ in range(steps):
        flush.zero_()
        a, b = ev(), ev()
        a.record(stream)
        out.append(body())
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    return ms, out


def ours_arm(args):
    import torch
    rank, world, local = dist_info()
    dist = init_dist(world)
    torch.cuda.set_device(local)
    import stratum_hyperdetail_b200 as sb
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    sb.lib()

    names = list(args.poses)
    views = []
    for name in names:
        p = POSES[name]
        v = View(WIDTH, HEIGHT)
        v.set_pose(SEED, p["origin"], p["pos"], p["yaw"], p["pitch"])
        views.append(v)
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    rays_per_step = WIDTH * HEIGHT * len(views)

    # -- 1. the plain per-frame drop-in path (reference launch sequence and shapes)
    trace_plain = np.zeros(len(views))

    def plain_step():
        te = [(ev(), ev()) for _ in views]
        n = sum(v.frame_parts(0.0, stream, te[i]) for i, v in enumerate(views))
        return n, te

    for _ in range(args.warmup):
        plain_step()
    plain_ms, plain_out = timed_steps(torch, stream, args.steps, flush, plain_step)
    for _, te in plain_out:
        trace_plain += np.array([x.elapsed_time(y) for x, y in te])
    plain_value = rays_per_step * args.steps / (sum(plain_ms) * 1e-3)
    per_pose = {n: WIDTH * HEIGHT * args.steps / (trace_plain[i] * 1e-3) for i, n in enumerate(names)}

    # -- 2. the batched path: every view in one launch per kernel, autotuned
    batch = Batch(views)
    batch.frame()
    tune_ms = batch.autotune()
    tune = {"threads": batch.tune.threads, "grab": batch.tune.grab, "order": batch.tune.order,
            "trace_ms": tune_ms}
    call, P, s = sb.call, sb.ptr, stream.cuda_stream

    def batch_step():
        t0, t1 = ev(), ev()
        call("stratum_stepViews", P(batch.table), batch.n, s)
        batch.refresh(stream)
        t0.record(stream)
        batch.trace(stream)
        t1.record(stream)
        batch.shade(stream)
        return t0, t1

    for _ in range(args.warmup):
        batch_step()
    eager_ms, eager_out = timed_steps(torch, stream, args.steps, flush, batch_step)
    trace_batch_ms = sum(a.elapsed_time(b) for a, b in eager_out)
    eager_value = rays_per_step * args.steps / (sum(eager_ms) * 1e-3)

    # -- 3. the same batched frame captured once as a CUDA graph and replayed (headline)
    graph_ok = True
    try:
        batch.capture()
    except Exception as e:  # pragma: no cover - reported, not hidden
        graph_ok = False
        graph_err = repr(e)
    if graph_ok:
        for _ in range(args.warmup):
            batch.replay()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            wall0 = time.perf_counter()
            step_ms, _ = timed_steps(torch, stream, args.steps, flush, batch.replay)
            torch.cuda.synchronize()
            wall = time.perf_counter() - wall0
        launches = batch.launches_per_frame * args.steps
        path = "batched: all views per launch, persistent tile queue, CUDA graph replay"
    else:
        with ClockSampler(local) as clocks:
            wall0 = time.perf_counter()
            step_ms, _ = timed_steps(torch, stream, args.steps, flush, lambda: batch.frame(stream))
            wall = time.perf_counter() - wall0
        launches = batch.launches_per_frame * args.steps
        path = "batched: all views per launch, persistent tile queue (eager; graph capture failed)"
    elapsed = sum(step_ms) * 1e-3
    if dist:
        t = torch.tensor([elapsed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = rays_per_step * args.steps * world / elapsed

    # -- roofline of the dominant kernel (traceViewsK): algorithmic FP32 ops / its event time
    peak = issue_peak(torch, sb)
    trace_ops = sum(OPS_PER_RAY[n][1] for n in names) * WIDTH * HEIGHT * args.steps
    achieved = trace_ops / (trace_batch_ms * 1e-3)
    traffic = (TRACE_DRAM_BYTES_PER_RAY * rays_per_step) if TRACE_DRAM_BYTES_PER_RAY else None
    whole_ops = sum(OPS_PER_RAY[n][0] for n in names) * WIDTH * HEIGHT * args.steps
    roofline = {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": "traceViewsK (one launch per step)",
                "peak_source": "measured in this run (stratum_issueProbe: FP32 lane ops/s, no FMA)",
                "ops_source": "algorithmic FP32 ops per ray from the reference source (oracle/count_work.py)",
                "path_frac": whole_ops / elapsed * world / world / peak,
                "plain_trace_frac": trace_ops / (trace_plain.sum() * 1e-3) / peak}

    # -- e2e: the batched C-ABI call with the step's inputs from pinned host memory and RGBA8 back
    host_in = [torch.zeros(32, dtype=torch.float32).pin_memory() for _ in views]
    host_px = [torch.empty(WIDTH * HEIGHT, dtype=torch.int32).pin_memory() for _ in views]

    def e2e_step():
        for i, v in enumerate(views):
            v.I.copy_(host_in[i], non_blocking=True)
        batch.frame(stream)
        for i, v in enumerate(views):
            host_px[i].copy_(v.Pixels, non_blocking=True)

    e2e_step()
    e2e_ms, _ = timed_steps(torch, stream, max(3, args.steps // 2), flush, e2e_step)
    h2d = sum(t.numel() * 4 for t in host_in)
    d2h = sum(t.numel() * 4 for t in host_px)
    e2e_value = rays_per_step * len(e2e_ms) * world / (sum(e2e_ms) * 1e-3)

    # -- serving: continuous batching over resident sessions (open-loop Poisson arrivals)
    serving = None
    n_views = len(views)
    tune_t = (batch.tune.threads, batch.tune.grab, batch.tune.order)
    batch.graph = None  # release the graph (and, below, the views) before serving and the process group
    del batch, views
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if args.serve_seconds > 0 and world == 1:
        serving = {
            "mixed_256_sessions": serve_poisson(200.0, 256, args.serve_seconds, (768, 1024, 1600, 1920), 150 << 30,
                                                args.serve_views, 3, tune_t),
            "sessions_64_at_1600x900": serve_poisson(200.0, 64, args.serve_seconds, (1600,), 150 << 30,
                                                     args.serve_views, 3, tune_t, seed=2),
            "plain_path_per_view_ms": sum(plain_ms) / args.steps / len(names),
        }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ol, lib, kind = cpu_lib()
        rays, times, nthreads = cpu_sample(ol, lib, args.cpu_rows, steps=1)
        cpu = {"value": rays / times[0], "unit": "rays/s", "cores": nthreads, "kind": kind,
               "sample": f"{args.cpu_rows}-row band at mid-frame of each of the 6 poses at 1600x900 ({rays} rays), "
                         "trace + shade + resolve of the band"}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural world, fixed poses)",
            "config": {"workload": "plain single-view frame 1600x900, seed 0x5EED, six poses, one sample per view "
                                   "per step accumulating toward 64",
                       "width": WIDTH, "height": HEIGHT, "views_per_step": n_views,
                       "poses": {n: POSES[n] for n in names}, "path": path, "tune": tune,
                       "l2": "flushed between timed steps (256 MiB write outside the timed region)",
                       "parallelism": f"replicas x{world}"},
            "plain_path": {"value": plain_value, "unit": "rays/s", "ms_per_step": sum(plain_ms) / args.steps,
                           "launches_per_step": plain_out[0][0],
                           "note": "reference launch structure: per view 15 trace + 15 shade strips of 64 rows"},
            "batched_eager": {"value": eager_value, "ms_per_step": sum(eager_ms) / args.steps},
            "batched_vs_plain": value / plain_value,
            "per_pose_trace_rays_per_s": per_pose,
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "rays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "call": "stratum_frameViews over the batch, pinned host input and RGBA8 readback"},
            "gpu_launches": launches, "clocks": clocks.summary(), "wall_s": wall, "serving": serving}
    if not graph_ok:
        line["graph_error"] = graph_err
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    args = parse(argv)
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
