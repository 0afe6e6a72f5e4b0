"""Benchmark: spectral paths/s of the hdcx CUDA integrator on B200.

One step = one Render call of the 1.0M-triangle heavy-geometry workload
(1920x1080, 64 spp, 8 bounces, lat-long HDR dome; seeded synthetic scene, see
hdcodex_b200/workloads.py): 398,131,200 spectral paths (pixels x spp x 3
wavelength lanes). With N ranks every rank renders its own sample range of the
same frame on its own GPU (weak scaling, no collective on the data path).

Printed JSON line:
  value       - spectral paths/s of all ranks, device time of the K timed
                renders (CUDA events on the tracer's stream, max over ranks),
                scene and image resident in HBM;
  e2e         - the same metric through the C ABI call a caller makes
                (hdcx_render) with the image copied to a pinned host buffer
                every step, wall clock around the call;
  roofline    - the closest-hit traversal kernel: algorithmic bytes per ray
                (32 B ray + 16 B hit + 80 B per wide node visited + 36 B per
                triangle tested, visits counted by a counting pass) over its
                CUDA-event time, against the measured HBM copy bandwidth;
  cpu_baseline- the CPU oracle on the host cores over rows spread evenly
                over the frame (cpu_sample_rows).
`--impl reference` times the reference's own integrator on the host cores, on
rank 0 only: its GLSL compiled as C++ (oracle/_ref, built from the reference's
sources by oracle/ref_build.py) when that library is present, else the
oracle's restatement; same workload and metric, the same rows as
cpu_baseline, a chunk of them per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "spectral paths/s"
UNIT = "spectral paths/s"
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hdcx", choices=["hdcx", "reference"])
    ap.add_argument("--workload", default="heavy",
                    choices=["heavy", "heavy-instanced", "box", "stress", "batch", "nrc", "cache-kernels"],
                    help="heavy: 1.0M triangles, 1920x1080, 64 spp (the headline); heavy-instanced: the same "
                         "shape with its spheres as 256 instances of four prototypes (two-level BVH); "
                         "box: 34-triangle closed box, "
                         "256x256, 16 spp; stress: 200k-triangle spectral stress scene, 1280x720, 256 spp; "
                         "batch: --jobs scenes of 10k-2M triangles rendered by hdcx_render_batch; "
                         "nrc: time to a relative XYZ RMSE on the stress scene, radiance cache vs plain; "
                         "cache-kernels: radiance-cache query and training throughput")
    ap.add_argument("--jobs", type=int, default=64, help="jobs of the batch workload")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="batch workload: launch the jobs on their streams instead of one captured CUDA graph")
    ap.add_argument("--ref-spp", type=int, default=4096, help="nrc workload: spp of the FP64 reference")
    ap.add_argument("--target-rmse", type=float, default=0.02, help="nrc workload: relative XYZ RMSE to reach")
    ap.add_argument("--chunk-spp", type=int, default=4, help="nrc workload: spp per progressive render call")
    ap.add_argument("--max-spp", type=int, default=4096, help="nrc workload: give up after this many spp")
    ap.add_argument("--nrc-prefix", default="2,1",
                    help="nrc workload: comma-separated prefix bounces of the cache arms (the first is `value`)")
    ap.add_argument("--nrc-spread", default="0.01",
                    help="nrc workload: comma-separated spread factors c of further cache arms that end paths by "
                         "the spread heuristic (prefix --nrc-spread-cap as the latest bounce); empty: none")
    ap.add_argument("--nrc-spread-cap", type=int, default=4,
                    help="nrc workload: latest bounce of the spread arms' paths")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default="",
                    help="wave_paths,trace_blocks_per_sm,shade_blocks_per_sm[,sort_hits[,sort_rays]] to use instead of "
                         "autotuning (to repeat a tuned run, e.g. under a profiler)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip hdcx_autotune (by default it picks wave and grid sizes before the warm-up; setup, "
                         "not timed)")
    ap.add_argument("--profile", action="store_true",
                    help="render exactly one frame and exit (for ncu launch lists and captures)")
    ap.add_argument("--width", type=int, default=0, help="override the workload width (profiling only)")
    ap.add_argument("--height", type=int, default=0, help="override the workload height (profiling only)")
    ap.add_argument("--spp", type=int, default=0, help="override the workload spp (profiling only)")
    return ap.parse_args()


WORKLOADS = {"heavy": "heavy_geometry", "heavy-instanced": "heavy_geometry", "box": "closed_box",
             "stress": "spectral_stress"}


def make_workload(name, args=None):
    """The named workload; --width/--height/--spp (profiling only) resize it."""
    from hdcodex_b200 import workloads
    make = getattr(workloads, WORKLOADS[name])
    overrides = {"instanced": True} if name == "heavy-instanced" else {}
    if args is not None:
        for key in ("width", "height", "spp"):
            if getattr(args, key):
                overrides[key] = getattr(args, key)
    return make(**overrides)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def traffic_from_profile(workload):
    """DRAM bytes per extension ray of the closest-hit kernel from the committed
    ncu summary of this workload (profiles/extend_kernel_traffic_<workload>.json),
    or None where no capture of it was made."""
    path = os.path.join(ROOT, "profiles", f"extend_kernel_traffic_{workload}.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", "-i", str(self.index),
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
               "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
               "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
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
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(s[0]) for s in self.samples if num(s[0])]
        mx = [num(s[1]) for s in self.samples if num(s[1])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier_sync(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(value, world):
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# The CPU sample: rows spread evenly over the frame, full width, at the
# workload's spp, about 6M spectral paths in all. cpu_baseline and the
# reference arm time the same rows, so the two CPU rates are comparable with
# each other and, since the rows cross the whole frame, with a full-frame
# GPU rate.
CPU_SAMPLE_PATHS = 6_000_000


def cpu_sample_rows(wl):
    """Row indices of the CPU sample: R rows at y = floor((i + 1/2) H / R)."""
    per_row = wl.width * wl.spp * 3
    rows = int(min(wl.height, max(1, round(CPU_SAMPLE_PATHS / per_row))))
    return [int((i + 0.5) * wl.height / rows) for i in range(rows)]


def describe_rows(wl, rows):
    shown = ", ".join(str(y) for y in rows[:6]) + (", ..." if len(rows) > 6 else "")
    return (f"{len(rows)} rows spread evenly over the {wl.width}x{wl.height} frame (y = {shown}), full width, "
            f"at {wl.spp} spp")


def render_rows(t, wl, rows, sample_index, threads):
    for y in rows:
        t.render(wl.camera, wl.width, wl.height, sample_index, wl.max_bounces, wl.spp, crop=(0, y, wl.width, y + 1),
                 threads=threads)


def cpu_baseline(wl, target_seconds, rank0=True):
    """The oracle on the host cores over the CPU sample (cpu_sample_rows),
    repeated until about target_seconds have passed."""
    import oracle as O
    O.build()
    t = O.OracleTracer()
    t.set_scene(wl.scene)
    threads = os.cpu_count() or 1
    rows = cpu_sample_rows(wl)
    passes, secs, rays = 0, 0.0, 0
    while passes == 0 or secs < target_seconds:
        t0 = time.perf_counter()
        for y in rows:
            t.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp, crop=(0, y, wl.width, y + 1),
                     threads=threads)
            rays += sum(t.last_counters)
        secs += time.perf_counter() - t0
        passes += 1
    paths = passes * len(rows) * wl.width * wl.spp * 3
    return {"value": paths / secs, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{describe_rows(wl, rows)}, {passes} pass(es): {paths} spectral paths in {secs:.1f} s; "
                      f"the same rows as the reference arm",
            "rays_per_s": rays / secs}


def traversal_roofline(tracers_and_workloads, peak, peak_kind):
    """Roofline of the closest-hit traversal kernel over untimed renders of
    the given (tracer, workload) pairs: node visits and triangle tests from a
    counting render, extension rays and extendKernel time from a stage-timed
    render; algorithmic bytes (32 B ray + 16 B hit + 80 B per wide node + 36 B
    per triangle) over the kernel's time, against the HBM copy peak."""
    from hdcodex_b200.tracer import PROFILE_COUNT_TRAVERSAL, PROFILE_STAGE_TIMES
    total_bytes, total_ms, rays, nodes, tris = 0.0, 0.0, 0, 0, 0
    for t, wl in tracers_and_workloads:
        t.set_profiling(PROFILE_COUNT_TRAVERSAL)
        t.render_device(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp)
        c = t.stats()
        t.set_profiling(PROFILE_STAGE_TIMES)
        t.render_device(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp)
        st = t.stats()
        t.set_profiling(0)
        r = max(c["extension_rays"], 1)
        per_ray = 32 + 16 + 80 * c["extension_node_visits"] / r + 36 * c["extension_triangle_tests"] / r
        total_bytes += per_ray * st["extension_rays"]
        total_ms += st["extend_ms"]
        rays += c["extension_rays"]
        nodes += c["extension_node_visits"]
        tris += c["extension_triangle_tests"]
    achieved = total_bytes / (total_ms / 1000.0) / 1e9 if total_ms > 0 else None
    return {"kernel": "extendKernel (closest-hit traversal)", "bound": "hbm", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
            "traffic": None, "nodes_per_ray": nodes / max(rays, 1), "triangles_per_ray": tris / max(rays, 1),
            "jobs_measured": len(tracers_and_workloads)}


def workload_config(wl, world):
    from hdcodex_b200 import workloads
    return {"workload": wl.name, "triangles": workloads.triangle_count(wl.scene), "width": wl.width,
            "height": wl.height, "spp": wl.spp, "max_bounces": wl.max_bounces, "spectral_lanes": 3,
            "spectral_paths_per_step_per_gpu": wl.spectral_paths,
            "l2": "inputs larger than L2 (scene + BVH + dome + per-wave path state)",
            "parallelism": f"replicas x{world}, disjoint sample ranges"}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return  # rank 0 alone times the CPU reference
    if args.workload == "batch":
        from hdcodex_b200 import workloads
        wl = workloads.batch_job(0)
    else:
        wl = make_workload(args.workload)
    import oracle as O
    if O.ref_available():
        t, kind = O.ReferenceTracer(), "reference"
    else:
        O.build()
        t, kind = O.OracleTracer(), "port"
    t.set_scene(wl.scene)
    threads = os.cpu_count() or 1
    # Each step renders one chunk of the CPU sample's rows, in turn: every
    # few consecutive steps cover the sample cpu_baseline times.
    rows = cpu_sample_rows(wl)
    chunk = max(1, len(rows) // 4)
    chunks = [rows[i:i + chunk] for i in range(0, len(rows), chunk)]
    for i in range(args.warmup):
        render_rows(t, wl, chunks[i % len(chunks)], i * wl.spp, threads)
    times, paths = [], 0
    for i in range(args.steps):
        step_rows = chunks[(args.warmup + i) % len(chunks)]
        t0 = time.perf_counter()
        render_rows(t, wl, step_rows, (args.warmup + i) * wl.spp, threads)
        times.append(time.perf_counter() - t0)
        paths += len(step_rows) * wl.width * wl.spp * 3
    value = paths / sum(times)
    sample = (f"{describe_rows(wl, rows)}; each step renders {chunk} of these rows in turn "
              f"(the rows cpu_baseline times)")
    if kind == "reference":
        sample += "; the reference's GLSL integrator compiled as C++, ray queries on a CPU BVH"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(wl, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_batch(args):
    """The multi-job workload: every step renders all jobs (each job's own
    resolution and spp) through hdcx_render_batch, with the images read back to
    pinned host memory; the serial loop of hdcx_render calls over the same
    jobs is timed beside it. Under torchrun the jobs are dealt round-robin to
    the ranks (total work fixed: strong scaling)."""
    import torch

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from hdcodex_b200 import PathTracer, render_batch, workloads

    from hdcodex_b200.multigpu import job_shard
    jobs = [workloads.batch_job(i) for i in job_shard(args.jobs, world, rank)]
    tracers = []
    for wl in jobs:
        t = PathTracer(local)
        t.set_scene(wl.scene)
        tracers.append(t)
    hosts = [torch.empty((wl.height, wl.width, 4), dtype=torch.float32, pin_memory=True) for wl in jobs]
    paths = sum(wl.spectral_paths for wl in jobs)
    # Launch tuning (setup, untimed): --tuning, else the autotuner's pick for
    # the job with the most paths, applied to every job.
    if args.tuning:
        knobs = [int(x) for x in args.tuning.split(",")] + [0, 0]
        tuning = {"wave_paths": knobs[0], "trace_blocks_per_sm": knobs[1], "shade_blocks_per_sm": knobs[2],
                  "sort_hits": knobs[3], "sort_rays": knobs[4]}
    elif args.autotune and jobs:
        big = max(range(len(jobs)), key=lambda k: jobs[k].spectral_paths)
        wl = jobs[big]
        tuned = tracers[big].autotune(wl.camera, wl.width, wl.height, wl.max_bounces, wl.spp)
        tuning = {k: tuned[k] for k in ("wave_paths", "trace_blocks_per_sm", "shade_blocks_per_sm", "sort_hits",
                                        "sort_rays")}
    else:
        tuning = None
    if tuning:
        for t in tracers:
            t.set_tuning(**tuning)

    def batch_step(step):
        spec = [(t, wl.camera, wl.width, wl.height, step * wl.spp, wl.max_bounces, wl.spp, h.data_ptr())
                for t, wl, h in zip(tracers, jobs, hosts)]
        return render_batch(spec, graph=args.graph)

    def serial_step(step):
        for t, wl, h in zip(tracers, jobs, hosts):
            t.render(wl.camera, wl.width, wl.height, step * wl.spp, wl.max_bounces, wl.spp, out=h.data_ptr())

    for i in range(args.warmup):
        batch_step(i)
    sampler = ClockSampler(local)
    barrier_sync(world)
    sampler.start()
    t0 = time.perf_counter()
    per_job_ms = [0.0] * len(jobs)
    for i in range(args.steps):
        res = batch_step(args.warmup + i)
        for k, r in enumerate(res):
            per_job_ms[k] += r["render_ms"]
    barrier_sync(world)
    batch_s = max_over_ranks(time.perf_counter() - t0, world)
    clocks = sampler.stop()
    # The serial loop gets its own warm-up: each tracer's first hdcx_render
    # allocates its path buffers (in the batch, the lanes' buffers are shared).
    for i in range(args.warmup):
        serial_step(args.warmup + args.steps + i)
    barrier_sync(world)
    t0 = time.perf_counter()
    for i in range(args.steps):
        serial_step(2 * args.warmup + args.steps + i)
    barrier_sync(world)
    serial_s = max_over_ranks(time.perf_counter() - t0, world)
    total_paths = float(paths)
    if world > 1:
        import torch.distributed as dist
        tp = torch.tensor([float(paths)], dtype=torch.float64, device="cuda")
        dist.all_reduce(tp)
        total_paths = float(tp.item())
    roofline, baseline = None, None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        # The traversal roofline over the first eight jobs' own renders.
        roofline = traversal_roofline(list(zip(tracers, jobs))[:8], peak, peak_kind)
        if world == 1 and not args.no_cpu_baseline:
            try:
                baseline = cpu_baseline(jobs[0], args.cpu_seconds)
                baseline["sample"] = "job 0 of the batch: " + baseline["sample"]
            except Exception as exc:  # reported, never required
                baseline = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                            "sample": f"failed: {exc}"}
    if rank == 0:
        value = total_paths * args.steps / batch_s
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * batch_s / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batch-{args.jobs}-jobs", "jobs": args.jobs,
                       "spectral_paths_per_step": total_paths,
                       "triangles": sum(workloads.triangle_count(wl.scene) for wl in jobs) if world == 1 else None,
                       "l2": "inputs larger than L2", "parallelism": f"jobs dealt round-robin to {world} GPU(s)",
                       "launch": "one CUDA graph per batch frame" if args.graph else "jobs on their own streams",
                       "tuning": tuning},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 48 * len(jobs),
                    "d2h_bytes_per_step": sum(wl.width * wl.height * 16 for wl in jobs)},
            "serial_loop": {"value": total_paths * args.steps / serial_s, "unit": UNIT,
                            "ms_per_step": 1000.0 * serial_s / args.steps},
            "batch_over_serial": serial_s / batch_s,
            "per_job_device_ms_rank0": [round(ms / args.steps, 2) for ms in per_job_ms],
            "roofline": roofline,
            "cpu_baseline": baseline,
            "clocks": clocks,
        }), flush=True)
    for t in tracers:
        t.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_nrc(args):
    """Time to --target-rmse relative XYZ RMSE (||X - X_ref|| / ||X_ref|| over
    all pixels and X, Y, Z) on the spectral-stress scene, the plain 8-bounce
    integrator against the radiance-cache form (2-bounce prefix, online
    training); X_ref = the plain integrator's FP64 XYZ at --ref-spp. Both arms
    render progressively, --chunk-spp samples per call; the clock covers the
    render calls (training included), not the error evaluation."""
    import numpy as np
    import torch

    torch.cuda.set_device(0)
    from hdcodex_b200 import PathTracer, RadianceCache, workloads

    wl = workloads.spectral_stress()
    if args.width or args.height:
        wl = workloads.spectral_stress(width=args.width or wl.width, height=args.height or wl.height)
    w, h = wl.width, wl.height

    def xyz_mean(t):
        total, samples = t.read_xyz()
        return total / max(samples, 1)

    # One launch tuning for every tracer (reference, plain and cache arms):
    # --tuning, or the autotuner's pick for a plain render call of the arms'
    # shape (a tracer with a radiance cache attached cannot be autotuned).
    if args.tuning:
        knobs = [int(x) for x in args.tuning.split(",")] + [0, 0]
        tuning = {"wave_paths": knobs[0], "trace_blocks_per_sm": knobs[1], "shade_blocks_per_sm": knobs[2],
                  "sort_hits": knobs[3], "sort_rays": knobs[4]}
    else:
        with PathTracer(0) as t:
            t.set_scene(wl.scene)
            tuned = t.autotune(wl.camera, w, h, wl.max_bounces, args.chunk_spp)
        tuning = {k: tuned[k] for k in ("wave_paths", "trace_blocks_per_sm", "shade_blocks_per_sm", "sort_hits",
                                        "sort_rays")}

    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        t.set_tuning(**tuning)
        t0 = time.perf_counter()
        done = 0
        # Sample indices disjoint from the measured arms' (which start at 0).
        first = 1 << 22
        half = None
        while done < args.ref_spp:
            k = min(256, args.ref_spp - done)
            t.render_device(wl.camera, w, h, first + done, wl.max_bounces, k)
            done += k
            if half is None and done >= args.ref_spp // 2:
                half = t.read_xyz()
        ref_s = time.perf_counter() - t0
        total = t.read_xyz()
        reference = total[0] / total[1]
    ref_norm = float(np.linalg.norm(reference))
    # Noise floor of the reference: its two halves differ by about twice its own error.
    second = (total[0] - half[0]) / (total[1] - half[1])
    reference_noise = 0.5 * float(np.linalg.norm(half[0] / half[1] - second)) / ref_norm

    # 2^16 training path suffixes per render call (the config's per-frame
    # count), spread over the call's waves.
    wave = tuning.get("wave_paths") or (12 << 20)
    waves_per_call = max(1, -(-(w * h * args.chunk_spp * 3) // wave))
    training_paths = max(1024, (1 << 16) // waves_per_call)

    def converge(cache, prefix=2, spread=0.0):
        curve = []
        with PathTracer(0) as t:
            t.set_scene(wl.scene)
            t.set_tuning(**tuning)
            if cache is not None:
                t.set_radiance_cache(cache, prefix_bounces=prefix, training_paths=training_paths, train_steps=4)
                t.set_radiance_cache_spread(spread)
            elapsed, spp, err = 0.0, 0, float("inf")
            torch.cuda.synchronize()
            while spp < args.max_spp:
                t0 = time.perf_counter()
                t.render_device(wl.camera, w, h, spp, wl.max_bounces, args.chunk_spp)
                torch.cuda.synchronize()
                elapsed += time.perf_counter() - t0
                spp += args.chunk_spp
                err = float(np.linalg.norm(xyz_mean(t) - reference)) / ref_norm
                curve.append((spp, round(elapsed, 4), round(err, 5)))
                if err < args.target_rmse:
                    break
            stats = t.radiance_cache_stats() if cache is not None else None
        reached = err < args.target_rmse
        return {"seconds": elapsed if reached else None, "spp": spp, "final_rel_rmse": err, "reached": reached,
                "curve": curve[:: max(1, len(curve) // 24)] + curve[-1:], "cache_stats": stats}

    plain = converge(None)

    def ms_per_spp(max_bounces, spp=32):
        # Cost of a sample of the plain integrator with paths cut after
        # `max_bounces` bounces. A cache arm whose paths end at bounce p
        # traces p + 1 extension rounds (the last finds the vertex that
        # queries the cache) and shades p full vertices: its cost lies between
        # the cuts after p and after p + 1 bounces, plus the cache's queries
        # and training.
        with PathTracer(0) as t:
            t.set_scene(wl.scene)
            t.set_tuning(**tuning)
            t.render_device(wl.camera, w, h, 0, max_bounces, args.chunk_spp)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(0, spp, args.chunk_spp):
                t.render_device(wl.camera, w, h, k, max_bounces, args.chunk_spp)
            torch.cuda.synchronize()
            return 1e3 * (time.perf_counter() - t0) / spp

    cost_bounds = {"plain_8_bounces": ms_per_spp(wl.max_bounces), "plain_cut_after_3": ms_per_spp(3),
                   "plain_cut_after_2": ms_per_spp(2), "plain_cut_after_1": ms_per_spp(1)}
    prefixes = [int(x) for x in str(args.nrc_prefix).split(",") if x.strip()]
    arms = {}
    for prefix in prefixes:
        with RadianceCache(0) as cache:
            arms[prefix] = converge(cache, prefix)
            arms[prefix]["prefix_bounces"] = prefix
    spread_arms = {}
    for factor in [float(x) for x in str(args.nrc_spread).split(",") if x.strip()]:
        with RadianceCache(0) as cache:
            spread_arms[factor] = converge(cache, args.nrc_spread_cap, factor)
    cached = arms[prefixes[0]]
    ratio = (cached["seconds"] / plain["seconds"]) if (plain["seconds"] and cached["seconds"]) else None
    peak, peak_kind = measured_peaks()
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        t.set_tuning(**tuning)
        sized = workloads.spectral_stress(width=w, height=h, spp=args.chunk_spp)
        roofline = traversal_roofline([(t, sized)], peak, peak_kind)
    baseline = None
    if not args.no_cpu_baseline:
        # The oracle's rate on the stress scene's row sample, and the time it
        # would take to trace the plain arm's spp at that rate.
        try:
            baseline = cpu_baseline(workloads.spectral_stress(width=w, height=h, spp=args.chunk_spp), args.cpu_seconds)
            if plain["spp"] and baseline["value"]:
                baseline["projected_seconds_to_target"] = w * h * 3 * plain["spp"] / baseline["value"]
        except Exception as exc:
            baseline = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {exc}"}
    print(json.dumps({
        "metric": "time to 2% relative XYZ RMSE, radiance cache vs plain", "unit": "s",
        "value": cached["seconds"], "plain_seconds": plain["seconds"], "cache_over_plain": ratio,
        "higher_is_better": False, "n_gpus": 1, "dtype": "f32 path tracing, bf16 tensor-core MLP",
        "data": "synthetic",
        "config": {"workload": wl.name, "width": w, "height": h, "reference_spp": args.ref_spp,
                   "reference_seconds": ref_s, "reference_rel_noise": reference_noise,
                   "target_rel_rmse": args.target_rmse, "chunk_spp": args.chunk_spp,
                   "cache": "16 levels x 2 features, 2^19 entries/level fp16; MLP 64x4 ReLU bf16; "
                            f"prefix {prefixes[0]} bounces; {training_paths} training paths per wave "
                            f"({waves_per_call} wave(s) per call: 2^16 per call), 4 Adam steps per wave",
                   "tuning": tuning},
        "roofline": roofline, "cpu_baseline": baseline,
        "plain": plain, "cache": cached,
        "cache_by_prefix": {str(k): {"seconds": v["seconds"], "spp": v["spp"], "final_rel_rmse": v["final_rel_rmse"],
                                     "ratio_to_plain": (v["seconds"] / plain["seconds"])
                                     if (v["seconds"] and plain["seconds"]) else None}
                            for k, v in arms.items()},
        "ms_per_spp": {"plain": 1e3 * plain["seconds"] / plain["spp"] if plain["seconds"] else None,
                       **{f"cache_prefix_{k}": 1e3 * v["seconds"] / v["spp"] if v["seconds"] else None
                          for k, v in arms.items()},
                       **{f"cache_spread_{k:g}": 1e3 * v["seconds"] / v["spp"] if v["seconds"] else None
                          for k, v in spread_arms.items()},
                       "bounds_without_cache": cost_bounds},
        "cache_by_spread": {f"c={k:g}, latest bounce {args.nrc_spread_cap}": {
            "seconds": v["seconds"], "spp": v["spp"], "final_rel_rmse": v["final_rel_rmse"],
            "ratio_to_plain": (v["seconds"] / plain["seconds"]) if (v["seconds"] and plain["seconds"]) else None,
            "queries": (v["cache_stats"] or {}).get("queries")}
            for k, v in spread_arms.items()},
    }), flush=True)


def run_cache_kernels(args):
    """Radiance-cache kernel throughput with the default cache (2^19 entries
    per level): queries of 2^21 records and training steps on 2^16 samples
    (Adam over all parameters included), CUDA events on the device, after
    --warmup untimed calls of each."""
    import numpy as np
    import torch

    torch.cuda.set_device(0)
    from hdcodex_b200 import RadianceCache

    rng = np.random.default_rng(0)

    def records(n):
        q = np.zeros((n, 12), np.float32)
        q[:, :3] = rng.uniform(0, 1, (n, 3))
        d = rng.normal(size=(n, 3))
        q[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
        q[:, 6:9] = -q[:, 3:6]
        q[:, 9] = rng.uniform(0, 1, n)
        q[:, 10] = rng.uniform(0, 1, n)
        return torch.from_numpy(q).cuda()

    nq, nt = 1 << 21, 1 << 16
    with RadianceCache(0) as cache:
        train_q, train_y = records(nt), torch.rand(nt, device="cuda") + 0.5
        query_q, out = records(nq), torch.empty(nq, device="cuda")
        for _ in range(max(args.warmup, 1)):
            cache.train(train_q.data_ptr(), train_y.data_ptr(), nt, 1)
            cache.query(query_q.data_ptr(), nq, out.data_ptr())
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        for _ in range(args.steps):
            cache.query(query_q.data_ptr(), nq, out.data_ptr())
        stop.record()
        torch.cuda.synchronize()
        query_ms = start.elapsed_time(stop) / args.steps
        start.record()
        for _ in range(args.steps):
            loss = cache.train(train_q.data_ptr(), train_y.data_ptr(), nt, 1)
        stop.record()
        torch.cuda.synchronize()
        train_ms = start.elapsed_time(stop) / args.steps
        flops_per_query = 2 * (4 * 64 * 64 + 16 * 64)
        print(json.dumps({
            "metric": "radiance-cache queries/s", "value": nq / (query_ms / 1000.0), "unit": "queries/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "dtype": "bf16 tensor-core MLP, fp16 hash grid, fp32 Adam", "data": "synthetic",
            "config": {"workload": "cache-kernels", "queries_per_call": nq, "samples_per_train_step": nt,
                       "grid_parameters": cache.grid_parameter_count},
            "query_ms": query_ms, "train_step_ms": train_ms, "last_loss": loss,
            "mlp_tflops_in_query": nq * flops_per_query / (query_ms / 1000.0) / 1e12,
        }), flush=True)


def run_hdcx(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from hdcodex_b200 import PathTracer, workloads
    from hdcodex_b200.tracer import PROFILE_COUNT_TRAVERSAL, PROFILE_STAGE_TIMES

    wl = make_workload(args.workload, args)
    tracer = PathTracer(local)
    tracer.set_scene(wl.scene)
    # Scene size and build cost (BVH bytes, set_scene wall time): the
    # instanced workload's two-level BVH against the flattened scene's.
    scene_info = tracer.scene_info()
    tuning = None
    if args.tuning:
        knobs = [int(x) for x in args.tuning.split(",")] + [0, 0]
        tracer.set_tuning(wave_paths=knobs[0], trace_blocks_per_sm=knobs[1], shade_blocks_per_sm=knobs[2],
                          sort_hits=knobs[3], sort_rays=knobs[4])
    elif args.autotune and not args.profile:
        tuning = tracer.autotune(wl.camera, wl.width, wl.height, wl.max_bounces, wl.spp)
    if args.profile:
        tracer.render_device(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp)
        print(json.dumps({"profile_frame": wl.name, "width": wl.width, "height": wl.height, "spp": wl.spp,
                          "stats": tracer.stats()}), flush=True)
        tracer.close()
        return
    paths_per_step = wl.spectral_paths

    from hdcodex_b200.multigpu import sample_range

    def sample_index(step):
        return sample_range(step, world, rank, wl.spp)

    # Warm-up, then one counting pass for the roofline's algorithmic bytes.
    for i in range(args.warmup):
        tracer.render_device(wl.camera, wl.width, wl.height, sample_index(i), wl.max_bounces, wl.spp)
    tracer.set_profiling(PROFILE_COUNT_TRAVERSAL)
    tracer.render_device(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp)
    counted = tracer.stats()
    tracer.set_profiling(PROFILE_STAGE_TIMES)

    # Timed region 1: device time, image resident in HBM.
    sampler = ClockSampler(local)
    barrier_sync(world)
    sampler.start()
    wall0 = time.perf_counter()
    render_ms, extend_ms, extend_launches, ext_rays, sh_rays, ss_rays, launches = 0.0, 0.0, 0, 0, 0, 0, 0
    shade_ms, shadow_ms = 0.0, 0.0
    for i in range(args.steps):
        tracer.render_device(wl.camera, wl.width, wl.height, sample_index(args.warmup + i), wl.max_bounces, wl.spp)
        st = tracer.stats()
        render_ms += st["render_ms"]
        extend_ms += st["extend_ms"]
        shade_ms += st["shade_ms"]
        shadow_ms += st["shadow_ms"]
        extend_launches += st["extend_launches"]
        ext_rays += st["extension_rays"]
        sh_rays += st["shadow_rays"]
        ss_rays += st["subsurface_rays"]
        launches += st["kernel_launches"]
    barrier_sync(world)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    tracer.set_profiling(0)
    total_ms = max_over_ranks(render_ms, world)
    value = paths_per_step * world * args.steps / (total_ms / 1000.0)

    # Timed region 2: end to end through hdcx_render with a pinned host image.
    host = torch.empty((wl.height, wl.width, 4), dtype=torch.float32, pin_memory=True)
    for i in range(max(1, args.warmup)):
        tracer.render(wl.camera, wl.width, wl.height, sample_index(i), wl.max_bounces, wl.spp, out=host.data_ptr())
    barrier_sync(world)
    e2e_wall = 0.0
    for i in range(args.steps):
        t0 = time.perf_counter()
        tracer.render(wl.camera, wl.width, wl.height, sample_index(args.warmup + i), wl.max_bounces, wl.spp,
                      out=host.data_ptr())
        e2e_wall += time.perf_counter() - t0
    barrier_sync(world)
    e2e_wall = max_over_ranks(e2e_wall, world)
    e2e_value = paths_per_step * world * args.steps / e2e_wall
    image = host.numpy()
    finite = bool(np.isfinite(image).all())

    # Roofline of the closest-hit traversal kernel.
    rays_c = max(counted["extension_rays"], 1)
    nodes_per_ray = counted["extension_node_visits"] / rays_c
    tris_per_ray = counted["extension_triangle_tests"] / rays_c
    bytes_per_ray = 32 + 16 + 80 * nodes_per_ray + 36 * tris_per_ray
    achieved_gbs = ext_rays * bytes_per_ray / (extend_ms / 1000.0) / 1e9 if extend_ms > 0 else None
    peak, peak_kind = measured_peaks()
    traffic = traffic_from_profile(args.workload)
    roofline = {
        "kernel": "extendKernel (closest-hit traversal)",
        "bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
        "frac": (achieved_gbs / peak) if achieved_gbs else None, "peak_source": peak_kind,
        # ncu DRAM bytes per extension ray (profiles/extend_kernel_traffic_heavy.json,
        # captured on a smaller frame) times this run's rays per launch.
        "traffic": (traffic["dram_bytes_per_ray"] * ext_rays / extend_launches
                    if traffic and extend_launches else None),
        "algorithmic_bytes_per_ray": bytes_per_ray, "nodes_per_ray": nodes_per_ray,
        "triangles_per_ray": tris_per_ray, "extend_ms_per_step": extend_ms / args.steps,
        "extend_launches_per_step": extend_launches / args.steps,
        "extend_share_of_step": extend_ms / render_ms if render_ms else None,
    }

    baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            baseline = cpu_baseline(wl, args.cpu_seconds)
        except Exception as exc:  # the baseline is reported, never required
            baseline = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                        "sample": f"failed: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(wl, world),
            "rays_per_s": (ext_rays + sh_rays + ss_rays) * world / (total_ms / 1000.0),
            "extension_rays_per_step": ext_rays / args.steps, "shadow_rays_per_step": sh_rays / args.steps,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 48,
                    "d2h_bytes_per_step": wl.width * wl.height * 16, "image_finite": finite},
            "gpu_launches": launches,
            "stage_ms_per_step": {"extend": extend_ms / args.steps, "shade": shade_ms / args.steps,
                                  "shadow": shadow_ms / args.steps,
                                  "other": (render_ms - extend_ms - shade_ms - shadow_ms) / args.steps},
            "roofline": roofline,
            "tuning": tuning if tuning is not None else tracer.tuning(),
            "scene": scene_info,
            "cpu_baseline": baseline,
            "clocks": clocks,
            "wall_s_timed": wall,
        }
        print(json.dumps(line), flush=True)
    tracer.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "nrc":
        run_nrc(args)
    elif args.workload == "cache-kernels":
        run_cache_kernels(args)
    else:
        run_hdcx(args)


if __name__ == "__main__":
    main()
