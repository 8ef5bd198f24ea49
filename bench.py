"""Benchmark of the wavefront hot path: Mrays/s of closest-hit + shadow rays.

Default workload (`--mode pt`): the wavefront path tracer on the 1920x1080 instanced scene
(200 instances of 8 seeded meshes, ~1.30M instanced triangles, materials Lambertian / Phong /
Cook-Torrance / glass / mirror, 16 triangle area lights + constant environment), 16 samples
per pixel, up to 8 bounces (max_path_len 9), Russian roulette from bounce 3. One step = one
frame rendered entirely on the GPU (sample generation, traversal, shading, shadow rays), its
bounce loop replayed as a CUDA graph. Scene data is resident in HBM; the path and shadow
queues (~285 B per path in flight, several GB) exceed the 126 MB L2. Before timing, the
autotuner picks the traversal kernel of each query class and the wavefront size (untimed).
`value` counts every closest-hit and shadow ray the frame traced.

`e2e`: the same frames through the public API with the image copied back to pinned host
memory every frame (the camera set-up goes host -> device per frame).
`--impl reference`: the reference's own PathTracer / TileScheduler / Scene / materials (its
C++ built in place as oracle/_ref) on all host cores, on a bounded image of the same scene,
with the oracle's CPU traversal behind its traversal entry points (the reference's AnyDSL
traversal library is not part of its tree). Its ray counts are the reference scheduler's own.
`--mode trace`: traversal kernels alone on fixed ray sets of the same frame (kernel tuning).

`serving` (single GPU; `--mode serve` alone): the request server against the same requests
served one at a time through the single-request path, on the same GPU with the same resident
scenes (12 sphere fields of 10k-2M triangles). Config 4: 256 renders submitted at once
(requests/s = 256 / makespan; latency = submission to image in host memory). Config 5:
Poisson arrivals of 1080p 1-spp frames and 64k-4M-ray batches (p50 / p99 latency).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "pt_1080p_16spp_8bounce_instanced_200x8"
METRIC = "Mrays/s closest+shadow"
SPP = 16
MAX_PATH_LEN = 9        # 8 continuation bounces (path vertices incl. camera and light)
RR_START = 3
CPU_SAMPLE = (240, 135)  # bounded CPU sample: 1/64 of the pixels, same spp and bounces
# DRAM bytes (read + write) per closest-hit ray inside this frame: 3,755 MB over the 78.3M
# rays of the 9 closest-hit launches of one frame of this workload (one wavefront of all
# samples), captured with
#   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum
#       --clock-control none -k regex:trace_persistent -s 54 -c 18
#       python bench.py --steps 1 --warmup 3 --no-cpu-baseline --no-serving --no-vcm --no-config3
#       --no-autotune --paths-in-flight 33177600
# (1 pass per launch). roofline.traffic scales it by the rays of an average launch.
CLOSEST_DRAM_BYTES_PER_RAY = 48.0
# Device queues per path in flight: two path queues (ray 32 B, pixel 4, RNG 8, throughput 16,
# bounce 4), hit 16, two shadow queues (ray 32, hit 16, pixel 4, contribution 16), grouping
# key 1 and permutation entry 4.
QUEUE_BYTES_PER_PATH = 2 * 64 + 16 + 2 * 68 + 5


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.first = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def mark(self):
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[max(self.first - 1, 0):]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the CPU baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def peak_hbm():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def trace_bytes(rays: int, work) -> int:
    """Algorithmic bytes of traversal launches: 32 B ray + 16 B hit per ray, 80 B per 8-wide
    node fetched, 48 B per triangle tested, 64 B per instance entered."""
    return 48 * rays + 80 * int(work[0]) + 48 * int(work[1]) + 64 * int(work[2])


def frame_roofline(pt, frame):
    """Closest-hit traversal inside path-traced frames: one frame with every traversal
    launch timed by CUDA events on the launching stream (the host-driven loop, so each launch
    is timed alone), one with the statistics variant (identical hits) for the node / triangle
    / instance counts. `frame(seed)` renders one frame. Returns (profile, work, GB/s)."""
    from imbatracer_b200 import native as N
    lib = N.load()
    prof = N.PtProfile()
    prof.events = 1
    lib.imbart_pt_set_profile(pt.ctx, C_ref(prof))
    frame(30_000)
    lib.imbart_pt_set_profile(pt.ctx, None)
    work = N.PtProfile()
    work.work = 1
    lib.imbart_pt_set_profile(pt.ctx, C_ref(work))
    frame(30_000)
    lib.imbart_pt_set_profile(pt.ctx, None)
    closest_bytes = trace_bytes(work.closest_rays, work.closest_work)
    achieved = closest_bytes / max(prof.closest_launches, 1) / (prof.closest_ms / max(prof.closest_launches, 1) * 1e-3) / 1e9
    return prof, work, achieved


def config3_roofline(torch, dev, stream, peak):
    """The same roofline on the config-3 scene (2M triangles, 400 displaced spheres, one
    level): path-traced 1280x720 frames at 4 spp, max_path_len 9, traversal kernels tuned on
    the scene's own rays first (untimed)."""
    import ctypes
    from imbatracer_b200 import native as N
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200.integrators import GpuScene, PathTracer
    lib = N.load()
    classes = (N.TRACE_CLOSEST | N.TRACE_COHERENT, N.TRACE_CLOSEST, N.TRACE_ANY)
    saved = []
    for flags in classes:
        v, r = ctypes.c_int(0), ctypes.c_int(0)
        lib.imbart_get_trace_class(flags, ctypes.byref(v), ctypes.byref(r))
        saved.append((flags, v.value, r.value, lib.imbart_get_trace_tri_batch(flags)))
    desc = G.config3()
    gs = GpuScene(desc, device=dev.index or 0)
    sets = make_wavefront(desc, gs.trace_scene, torch, dev, 99, shadow_from_bounce=True)
    ray_sets = [(rays, torch.zeros((rays.shape[0], 4), dtype=torch.int32, device=dev), flags)
                for (rays, _), flags in zip(sets, classes)]
    nw = gs.autotune_node_width(ray_sets, stream=stream)
    del sets, ray_sets
    pt = PathTracer(gs, max_path_len=MAX_PATH_LEN, rr_start=RR_START)
    image = torch.zeros((desc.camera.height, desc.camera.width, 3), dtype=torch.float32, device=dev)
    for k in range(2):
        pt.render(4, 500 + k, image=image, stream=stream)
    prof, work, achieved = frame_roofline(pt, lambda seed: pt.render(4, seed, image=image, stream=stream))
    torch.cuda.synchronize()
    out = {"workload": f"config 3: {desc.instanced_triangles} triangles, 1280x720 at 4 spp, max_path_len {MAX_PATH_LEN}",
           "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
           "closest_mrays_s": round(work.closest_rays / max(prof.closest_ms, 1e-9) / 1e3, 1),
           "bytes_per_ray": round(trace_bytes(work.closest_rays, work.closest_work) / max(work.closest_rays, 1), 1),
           "launches": int(prof.closest_launches), "node_width": nw["node_width"],
           "node_width_tuned_ms": {str(k): v for k, v in nw["ms"].items()},
           "tuned": {name: {"variant": t["variant"], "refill": t["refill"]}
                     for name, t in zip(("camera", "bounce", "shadow"), (nw["classes"][f] for f in classes))}}
    pt.close()
    for flags, v, r, b in saved:   # the main frame's tuning again for what follows
        lib.imbart_set_trace_class(flags, v, r)
        lib.imbart_set_trace_tri_batch(flags, b)
    return out


class _StdoutToStderr:
    """Sends file descriptor 1 to stderr while the reference's C++ code prints its progress, so
    that the bench's stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def reference_cpu(desc, steps, threads, w, h, seed=7):
    """The reference's own CPU path tracer on a bounded image; returns (Mrays/s, rays/step, s/step)."""
    from oracle import refwrap as R
    with _StdoutToStderr():
        rs = R.RefScene(desc)
        tot_rays, tot_s = 0, 0.0
        for k in range(steps):
            t0 = time.perf_counter()
            _, a, b = rs.render_pt_threads(w, h, SPP, MAX_PATH_LEN, seed + k, threads)
            tot_s += time.perf_counter() - t0
            tot_rays += a + b
        rs.close()
    return tot_rays / tot_s / 1e6, tot_rays // max(steps, 1), tot_s / max(steps, 1)


def job_totals(ms: float, units: float, device, world: int) -> tuple[float, float]:
    """Whole-job figures of a multi-rank timing: the slowest rank's device time (max over
    ranks) and the units all ranks processed (sum); the rank's own values when world == 1."""
    if world <= 1:
        return float(ms), float(units)
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms, float(units)], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(t[1])


def run_pt(args):
    import torch
    import torch.distributed as dist
    from imbatracer_b200 import native as N
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200.integrators import GpuScene, PathTracer

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = N.load()

    desc = G.config2()
    gs = GpuScene(desc, device=local)
    W, H = desc.camera.width, desc.camera.height
    stream = torch.cuda.current_stream(dev)
    # Autotuner (untimed): the node width of the scene, then the kernel configuration of each
    # query class on this scene's rays at that width.
    tuning = {}
    if not args.no_autotune:
        sets = make_wavefront(desc, gs.trace_scene, torch, dev, 4321, shadow_from_bounce=True)
        classes = (N.TRACE_CLOSEST | N.TRACE_COHERENT, N.TRACE_CLOSEST, N.TRACE_ANY)
        ray_sets = [(rays, torch.zeros((rays.shape[0], 4), dtype=torch.int32, device=dev), flags)
                    for (rays, _), flags in zip(sets, classes)]
        nw = gs.autotune_node_width(ray_sets, stream=stream)
        tuning["node_width"] = {"chosen": nw["node_width"],
                                "tuned_ms_all_classes": {str(k): v for k, v in nw["ms"].items()}}
        for name, flags in zip(("camera", "bounce", "shadow"), classes):
            t = nw["classes"][flags]
            tuning[name] = {"variant": t["variant"], "refill": t["refill"], "tri_batch": t["tri_batch"],
                            "speedup": round(t["default_ms"] / max(t["ms"], 1e-9), 3)}
        del sets, ray_sets
        torch.cuda.synchronize()
    pt = PathTracer(gs, max_path_len=MAX_PATH_LEN, rr_start=RR_START)
    if not args.no_autotune:
        # Wavefront size (paths in flight) for this frame shape, with the tuned kernels.
        if not args.paths_in_flight:
            wf = pt.autotune_wavefront(SPP, seed_base=777, stream=stream)
            tuning["wavefront"] = {"paths_in_flight": pt.max_paths,
                                   "ms_per_frame": {str(k): round(v, 2) for k, v in wf.items()}}
        torch.cuda.synchronize()
    if args.paths_in_flight:
        pt.max_paths = args.paths_in_flight
    image = torch.zeros((H, W, 3), dtype=torch.float32, device=dev)
    base_seed = 1000 * (rank + 1)

    def frame(k):
        pt.render(SPP, base_seed + k, image=image, stream=stream)
        return int(pt.last_stats[0] + pt.last_stats[1])

    clocks = ClockSampler(local)
    clocks.start()
    for k in range(args.warmup):
        frame(k)
    torch.cuda.synchronize()
    clocks.mark()
    launches0 = lib.imbart_kernel_launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rays = 0
    for k in range(args.steps):
        rays += frame(args.warmup + k)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = lib.imbart_kernel_launch_count() - launches0
    ms = e0.elapsed_time(e1)
    ms_max, all_rays = job_totals(ms, rays, dev, world)

    # e2e through the public API: render + image copied to pinned host memory per frame.
    host_img = torch.empty((H, W, 3), dtype=torch.float32).pin_memory()
    for k in range(max(1, args.warmup // 2)):
        frame(10_000 + k)
        host_img.copy_(image, non_blocking=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    e2e_rays = 0
    for k in range(args.steps):
        e2e_rays += frame(20_000 + k)
        host_img.copy_(image, non_blocking=True)
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_ms, e2e_all = job_totals(q0.elapsed_time(q1), e2e_rays, dev, world)

    # The same frames under the reference's Russian-roulette policy (from bounce 0,
    # pt.cpp:53-57), which the reference arm runs: device time and end to end.
    pt.rr_start = 0
    for k in range(2):
        frame(40_000 + k)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    r0, r1, r2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    r0.record(stream)
    rr0_rays = 0
    for k in range(args.steps):
        rr0_rays += frame(50_000 + k)
    r1.record(stream)
    rr0_e2e_rays = 0
    for k in range(args.steps):
        rr0_e2e_rays += frame(60_000 + k)
        host_img.copy_(image, non_blocking=True)
    r2.record(stream)
    torch.cuda.synchronize()
    rr0_ms, rr0_all = job_totals(r0.elapsed_time(r1), rr0_rays, dev, world)
    rr0_e2e_ms, rr0_e2e_all = job_totals(r1.elapsed_time(r2), rr0_e2e_rays, dev, world)
    pt.rr_start = RR_START

    # Roofline of the dominant kernel (closest-hit traversal) inside the frame.
    prof, work, achieved = frame_roofline(pt, frame)
    torch.cuda.synchronize()
    closest_bytes = trace_bytes(work.closest_rays, work.closest_work)
    shadow_bytes = trace_bytes(work.shadow_rays, work.shadow_work)
    per_launch_bytes = closest_bytes / max(prof.closest_launches, 1)
    per_launch_ms = prof.closest_ms / max(prof.closest_launches, 1)
    peak, peak_src = peak_hbm()
    roof3 = config3_roofline(torch, dev, stream, peak) if world == 1 and not args.no_config3 else None

    if rank == 0:
        paths = min(pt.max_paths or (16 << 20), W * H * SPP)
        value = all_rays / (ms_max * 1e-3) / 1e6
        e2e_value = e2e_all / (e2e_ms * 1e-3) / 1e6
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            from oracle import refwrap as R
            if R.available():
                threads = os.cpu_count() or 1
                mr, rps, sps = reference_cpu(desc, 2, threads, *CPU_SAMPLE)
                cpu = {"value": round(mr, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                       "cpu_model": cpu_model(), "rr_start_bounce": 0,
                       "sample": f"{CPU_SAMPLE[0]}x{CPU_SAMPLE[1]} at {SPP} spp, max_path_len {MAX_PATH_LEN} "
                                 f"(1/64 of the frame's pixels), 2 frames, {rps} rays/frame: the reference's "
                                 f"PathTracer+TileScheduler ({threads} tile threads) with the oracle CPU traversal"}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator, per-pixel MWC64X seeding)",
            "config": {"workload": WORKLOAD, "resolution": f"{W}x{H}", "spp": SPP, "max_path_len": MAX_PATH_LEN,
                       "rr_start_bounce": RR_START, "instances": len(desc.instances), "meshes": len(desc.meshes),
                       "instanced_triangles": desc.instanced_triangles, "lights": len(desc.lights) + 1,
                       "rays_per_step": int(all_rays / world / args.steps),
                       "l2": f"path + shadow queues larger than L2 (~{QUEUE_BYTES_PER_PATH * paths / 1e9:.1f} GB "
                             f"for {paths} paths in flight); the scene itself (8-wide BVH ~11 MB, triangles, "
                             f"instances) stays L2-resident",
                       "parallelism": f"replicas x{world} (independent frames per GPU, different seeds)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": int(CLOSEST_DRAM_BYTES_PER_RAY * work.closest_rays
                                        / max(prof.closest_launches, 1)),
                         "traffic_unit": "bytes per launch (ncu capture, scaled by rays per launch)",
                         "kernel": "trace_persistent (closest hit) inside the frame", "peak_source": peak_src,
                         "bytes_per_launch": int(per_launch_bytes), "launch_ms": round(per_launch_ms, 4),
                         "launches": int(prof.closest_launches),
                         "bytes_per_ray": round(closest_bytes / max(work.closest_rays, 1), 1),
                         "shadow": {"ms": round(prof.shadow_ms, 3), "launches": int(prof.shadow_launches),
                                    "achieved_gbs": round(shadow_bytes / max(prof.shadow_ms, 1e-9) / 1e6, 1),
                                    "bytes_per_ray": round(shadow_bytes / max(work.shadow_rays, 1), 1)},
                         "trace_share_of_frame": round((prof.closest_ms + prof.shadow_ms) / (ms_max / args.steps), 3),
                         "closest_mrays_s": round(work.closest_rays / max(prof.closest_ms, 1e-9) / 1e3, 1),
                         "shadow_mrays_s": round(work.shadow_rays / max(prof.shadow_ms, 1e-9) / 1e3, 1)},
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 16 * 4 + 12,
                    "d2h_bytes_per_step": W * H * 12},
            "equal_policy": {
                "rr_start_bounce": 0, "unit": "Mrays/s",
                "value": round(rr0_all / (rr0_ms * 1e-3) / 1e6, 2),
                "ms_per_step": round(rr0_ms / args.steps, 2),
                "e2e": round(rr0_e2e_all / (rr0_e2e_ms * 1e-3) / 1e6, 2),
                "rays_per_step": int(rr0_all / world / args.steps),
                "note": "the same frames with Russian roulette from bounce 0, the reference's policy "
                        "(pt.cpp:53-57) and the reference arm's; the headline value uses the workload's "
                        "roulette from bounce 3"},
            "roofline_config3": roof3,
            "gpu_launches": int(launches),
            "autotune": tuning,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        if world == 1 and not args.no_serving:
            line["serving"] = run_serving()
        if world == 1 and not args.no_vcm:
            line["vcm_family"] = run_vcm()
            line["vcm_family"]["config3_spec"] = run_vcm_spec()
            if not args.no_cpu_baseline:
                from oracle import refwrap as R
                if R.available():
                    line["vcm_family"]["cpu_baseline"] = reference_vcm_cpu(os.cpu_count() or 1)
        if world == 1 and not args.no_config1:
            from oracle import refwrap as R
            line["config1"] = run_config1(cpu_threads=(os.cpu_count() or 1)
                                          if not args.no_cpu_baseline and R.available() else 0)
        print(json.dumps(line), flush=True)
    pt.close()
    gs.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def C_ref(s):
    import ctypes
    return ctypes.byref(s)


def run_reference(args):
    """The reference's own CPU path tracer (oracle/_ref) on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import refwrap as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref.so was not built (the reference "
                                                              "tree was absent when build() ran)"}))
        return
    from imbatracer_b200 import scenegen as G
    desc = G.config2()
    threads = os.cpu_count() or 1
    with _StdoutToStderr():
        rs = R.RefScene(desc)
    for k in range(args.warmup):
        rs.render_pt_threads(60, 34, SPP, MAX_PATH_LEN, 99 + k, threads)
    tot, el = 0, 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        _, a, b = rs.render_pt_threads(*CPU_SAMPLE, SPP, MAX_PATH_LEN, 7 + k, threads)
        el += time.perf_counter() - t0
        tot += a + b
    value = tot / el / 1e6
    sample = (f"{CPU_SAMPLE[0]}x{CPU_SAMPLE[1]} at {SPP} spp per step (1/64 of the 1080p frame), "
              f"{tot // max(args.steps, 1)} rays/step counted by the reference scheduler")
    line = {"metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "impl": "reference",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(el / args.steps * 1e3, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": WORKLOAD, "sample": sample, "max_path_len": MAX_PATH_LEN, "rr_start_bounce": 0,
                       "reference": "PathTracer/TileScheduler/Scene/materials of the reference built in place "
                                    "(oracle/_ref); traversal = the oracle's CPU restatement"},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                             "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# Serving: the request server (batched) against the same requests one at a time (plain)
# ---------------------------------------------------------------------------------------
SERVE_MAX_PATH_LEN = 5        # 4 bounces, as the sphere-field renders
SERVE_PATHS = int(os.environ.get("IMBART_SERVE_PATHS", 4 << 20))   # paths per merged (and single-request) wavefront
SERVE_BUDGET = 120 << 30      # device pool of the batched server (config 5's HBM budget)


HOST_BUILD_S: list = []      # host SBVH build + layout time of each serving scene


def serve_scenes():
    from imbatracer_b200 import scene as S
    from imbatracer_b200 import scenegen as G
    descs = G.config4_scenes()
    out = []
    HOST_BUILD_S.clear()
    for d in descs:
        t0 = time.perf_counter()
        out.append((d, S.build_traversal_data(d.meshes, d.instances)))
        HOST_BUILD_S.append(time.perf_counter() - t0)
    return out


def admission_times(scenes):
    """Scene admission: registering each serving scene with its traversal arrays built on the
    GPU (imbart_server_add_scene_gpu_build) and serving a first 64x64 frame on it (upload into
    the pool), beside the host SBVH build that the other registration path needs."""
    from imbatracer_b200.serving import Server
    srv = Server(mode="batched", hbm_budget=SERVE_BUDGET, max_paths=SERVE_PATHS)
    gpu_ms, first_ms = [], []
    for d, _ in scenes:
        sid = srv.add_scene(d, gpu_build=True)
        gpu_ms.append(srv.last_build_ms)
        t0 = time.perf_counter()
        t, _ = srv.submit_render(sid, d.camera, 64, 64, 1, SERVE_MAX_PATH_LEN, 1)
        srv.wait(t)
        first_ms.append((time.perf_counter() - t0) * 1e3)
    srv.close()
    tris = [d.instanced_triangles for d, _ in scenes]
    out = {"scene_triangles": tris, "gpu_build_ms": [round(v, 1) for v in gpu_ms],
           "first_frame_ms": [round(v, 1) for v in first_ms],
           "gpu_build_total_ms": round(sum(gpu_ms), 1)}
    if len(HOST_BUILD_S) == len(scenes):
        out["host_build_s"] = [round(v, 2) for v in HOST_BUILD_S]
        out["host_build_total_s"] = round(sum(HOST_BUILD_S), 2)
    return out


def _percentile(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


def serve_arm(mode, scenes, jobs, open_loop, ray_buf=None, hit_buf=None):
    """Runs `jobs` through a server of `mode`; returns latency / throughput figures."""
    import ctypes
    from imbatracer_b200 import native as N
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200.serving import Server
    srv = Server(mode=mode, hbm_budget=SERVE_BUDGET, max_paths=SERVE_PATHS)
    ids = [srv.add_scene(d, td) for d, td in scenes]
    # Warm-up: every scene once (uploads it), so that both arms start with resident scenes.
    warm = [srv.submit_render(ids[k], scenes[k][0].camera, 64, 64, 1, SERVE_MAX_PATH_LEN, 1) for k in range(len(ids))]
    vcm_sides = [j.width for j in jobs if isinstance(j, G.RenderJob) and j.integrator != "pt"]
    if vcm_sides:
        # One frame of the largest VCM-family size per VCM lane (4 in batched mode), so that
        # every lane's buffers have their final size before the timed region.
        side = max(vcm_sides)
        warm += [srv.submit_vcm(ids[0], scenes[0][0].camera, side, side, "vcm", max_path_len=SERVE_MAX_PATH_LEN)
                 for _ in range(4)]
    for t, _ in warm:
        srv.wait(t)
    s0 = srv.stats()
    images = {}
    for j in jobs:
        if isinstance(j, G.RenderJob) and (j.width, j.height) not in images:
            images[(j.width, j.height)] = np.zeros((j.height, j.width, 3), np.float32)
    tickets = []
    t_start = time.perf_counter()
    for j in jobs:
        if open_loop:
            delay = t_start + j.arrival_s - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
        if isinstance(j, G.RenderJob) and j.integrator != "pt":
            # BPT / VCM: spp iterations of one camera sample per pixel and width*height/2 light paths.
            cam = scenes[j.scene][0].camera
            t, _ = srv.submit_vcm(ids[j.scene], cam, j.width, j.height, j.integrator, iterations=j.spp,
                                  max_path_len=SERVE_MAX_PATH_LEN, light_seed=j.seed, camera_seed=j.seed ^ 0x5BD1E995,
                                  image=images[(j.width, j.height)])
        elif isinstance(j, G.RenderJob):
            cam = scenes[j.scene][0].camera
            t, _ = srv.submit_render(ids[j.scene], cam, j.width, j.height, j.spp, SERVE_MAX_PATH_LEN, j.seed,
                                     image=images[(j.width, j.height)])
        else:
            off = j.seed % (len(ray_buf) - j.count + 1)
            t = srv.lib.imbart_server_submit_rays(srv.h, ids[j.scene], N.ptr(ray_buf) + 32 * off,
                                                  N.ptr(hit_buf) + 16 * off, j.count, j.flags)
            assert t > 0
        tickets.append((t, j))
    res = [(srv.wait(t), j) for t, j in tickets]
    s1 = srv.stats()
    srv.close()
    assert all(r["status"] == 0 for r, _ in res)
    lat = [r["done_ms"] - r["submit_ms"] for r, _ in res]
    first = min(r["submit_ms"] for r, _ in res)
    last = max(r["done_ms"] for r, _ in res)
    renders = [r["done_ms"] - r["submit_ms"] for r, j in res if isinstance(j, G.RenderJob)]
    batches = [r["done_ms"] - r["submit_ms"] for r, j in res if not isinstance(j, G.RenderJob)]
    rays = (s1["closest_rays"] - s0["closest_rays"]) + (s1["shadow_rays"] - s0["shadow_rays"]) + \
           (s1["batch_rays"] - s0["batch_rays"])
    span_s = (last - first) * 1e-3
    out = {"requests_per_s": round(len(res) / span_s, 2), "makespan_s": round(span_s, 3),
           "p50_ms": round(_percentile(lat, 50), 2), "p99_ms": round(_percentile(lat, 99), 2),
           "mrays_s": round(rays / span_s / 1e6, 1), "waves": s1["waves"] - s0["waves"]}
    if renders and batches:
        out["render_p99_ms"] = round(_percentile(renders, 99), 2)
        out["batch_p99_ms"] = round(_percentile(batches, 99), 2)
    return out


# ---------------------------------------------------------------------------------------
# VCM family: iterations of VCM / PPM / BPT on the 2M-triangle sphere field (config 3)
# ---------------------------------------------------------------------------------------
VCM_W, VCM_H = 1280, 720
VCM_LIGHT_PATHS = 1 << 20
VCM_MAX_PATH_LEN = 8


def run_vcm(iterations=4, warmup=2, algos=("vcm", "ppm", "bpt")):
    """Device time per iteration (light pass + camera pass, one camera sample per pixel)."""
    import torch
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200.integrators import GpuScene, VcmIntegrator
    desc = G.config3(width=VCM_W, height=VCM_H)
    gs = GpuScene(desc)
    out = {"workload": f"config 3: {desc.instanced_triangles} triangles (400 displaced spheres), {VCM_W}x{VCM_H}, "
                       f"{VCM_LIGHT_PATHS} light paths and 1 camera sample per pixel per iteration, max path "
                       f"length {VCM_MAX_PATH_LEN}, 1 connection, 10 nearest photons, radius 2 pixel sizes "
                       f"shrinking as iteration^-1/8",
           "iterations": iterations, "warmup": warmup}
    for algo in algos:
        vi = VcmIntegrator(gs, algo, VCM_W, VCM_H, spp=1, max_path_len=VCM_MAX_PATH_LEN,
                           light_path_count=VCM_LIGHT_PATHS, num_connections=1, num_knn=10, radius_factor=2.0)
        image = torch.zeros((VCM_H, VCM_W, 3), dtype=torch.float32, device="cuda")
        for k in range(warmup):
            vi.render(k + 1, 11 + k, 101 + k, 0x9E3779B9, image=image)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rays, vertices = 0, 0
        for k in range(iterations):
            vi.render(warmup + k + 1, 1000 + k, 2000 + k, 0x9E3779B9, image=image)
            rays += int(vi.last_stats[0] + vi.last_stats[1])
            vertices += N_light_vertices(vi)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / iterations
        out[algo] = {"ms_per_iteration": round(ms, 2), "mrays_s": round(rays / iterations / (ms * 1e-3) / 1e6, 1),
                     "rays_per_iteration": rays // iterations, "light_vertices": vertices // iterations,
                     "pixel_size": round(vi.pixel_size, 5)}
        vi.close()
    gs.close()
    return out


def run_vcm_spec(iterations=64, warmup=2, algos=("vcm", "ppm")):
    """Config 3 at its own photon-grid parameters: 2^22 buckets, cell size = merge radius,
    r0 = 0.5 % of the scene diagonal shrinking as r_i = r0 * i^(-1/3), 64 iterations of 1M
    light paths and one camera sample per pixel (device time per iteration). Then the grid
    alone on the last iteration's light vertices: build time and k-nearest queries at every
    vertex (the split the CPU baseline reports)."""
    import torch
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200.hashgrid import HashGrid
    from imbatracer_b200.integrators import GpuScene, VcmIntegrator
    desc = G.config3(width=VCM_W, height=VCM_H)
    lo, hi = G.scene_box(desc)
    diag = float(np.linalg.norm(hi.astype(np.float64) - lo))
    r0 = 0.005 * diag
    gs = GpuScene(desc)
    out = {"workload": f"config 3 at its grid parameters: {desc.instanced_triangles} triangles, {VCM_W}x{VCM_H}, "
                       f"{VCM_LIGHT_PATHS} light paths and 1 camera sample per pixel per iteration, max path length "
                       f"{VCM_MAX_PATH_LEN}, 10 nearest photons, 2^22 buckets, cell = r, r0 = 0.005 x diagonal "
                       f"({r0:.4f}), r_i = r0 i^(-1/3)", "iterations": iterations, "warmup": warmup}
    last_cache = None
    for algo in algos:
        vi = VcmIntegrator(gs, algo, VCM_W, VCM_H, spp=1, max_path_len=VCM_MAX_PATH_LEN,
                           light_path_count=VCM_LIGHT_PATHS, num_connections=1, num_knn=10, base_radius=r0,
                           radius_exponent=1.0 / 3.0, grid_cell_factor=1.0, grid_table_size=1 << 22)
        image = torch.zeros((VCM_H, VCM_W, 3), dtype=torch.float32, device="cuda")
        for k in range(warmup):
            vi.render(k + 1, 11 + k, 101 + k, 0x9E3779B9, image=image)
        image.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rays = 0
        for k in range(iterations):
            vi.render(k + 1, 1000 + k, 2000 + k, 0x9E3779B9, image=image)
            rays += int(vi.last_stats[0] + vi.last_stats[1])
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / iterations
        vertices = N_light_vertices(vi)
        radius = vi.begin_iteration(iterations)[0]
        out[algo] = {"ms_per_iteration": round(ms, 2), "mrays_s": round(rays / iterations / (ms * 1e-3) / 1e6, 1),
                     "rays_per_iteration": rays // iterations, "light_vertices": vertices,
                     "radius_last_iteration": round(radius, 5)}
        if last_cache is None:
            vi.render(iterations, 1000, 2000, 0x9E3779B9, image=image)
            last_cache = (vi.light_vertices(), radius)
        vi.close()
    gs.close()
    if last_cache is not None and len(last_cache[0]):
        pos = torch.from_numpy(np.ascontiguousarray(last_cache[0][:, :3])).cuda()
        grid = HashGrid(0)
        grid.build(pos, last_cache[1], 1.0, 1 << 22)
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        for _ in range(10):
            grid.build(pos, last_cache[1], 1.0, 1 << 22)
        e1.record()
        ids, cnt = grid.query(pos, 10)
        e2.record()
        torch.cuda.synchronize()
        out["grid"] = {"photons": int(pos.shape[0]), "build_ms": round(e0.elapsed_time(e1) / 10, 3),
                       "queries": int(pos.shape[0]), "query_ms": round(e1.elapsed_time(e2), 3),
                       "mqueries_s": round(pos.shape[0] / (e1.elapsed_time(e2) * 1e-3) / 1e6, 1),
                       "note": "cell = r, 2^22 buckets, r of the last iteration; k = 10 nearest within r at "
                               "every light vertex (batched query API, one warp per query)"}
        grid.close()
    return out


def reference_vcm_cpu(threads: int) -> dict:
    """The reference's own VCMIntegrator (oracle/_ref) on the config-3 scene, one iteration
    at the reference's photon-grid parameters (cell 2r, 2n buckets, r = 2 pixel sizes: its
    HashGrid fixes them), on all host threads: light pass, camera pass, and the grid alone
    (rebuild; one k-nearest query at every light vertex)."""
    from imbatracer_b200 import scenegen as G
    from oracle import refwrap as R
    desc = G.config3(width=VCM_W, height=VCM_H)
    with _StdoutToStderr():
        rs = R.RefScene(desc)
        R.load().imbart_ref_set_threads(threads, threads)
        v = R.RefVcm(rs, "vcm", VCM_W, VCM_H, light_path_count=VCM_LIGHT_PATHS, max_path_len=VCM_MAX_PATH_LEN)
        v.begin_iteration(1)
        t0 = time.perf_counter()
        v.light_pass(11)
        t1 = time.perf_counter()
        v.camera_pass(22)
        t2 = time.perf_counter()
        g = v.time_grid(2, threads)
        v.close()
        rs.close()
        R.load().imbart_ref_set_threads(1, 1)
    return {"kind": "reference", "cores": threads, "cpu_model": cpu_model(), "unit": "ms/iteration",
            "value": round((t2 - t0) * 1e3, 1), "light_pass_ms": round((t1 - t0) * 1e3, 1),
            "camera_pass_ms": round((t2 - t1) * 1e3, 1), "grid_build_ms": round(g["build_s"] * 1e3, 1),
            "queries": g["queries"], "query_ms": round(g["query_s"] * 1e3, 1),
            "mqueries_s": round(g["queries"] / max(g["query_s"], 1e-9) / 1e6, 3),
            "sample": f"one VCM iteration (iteration 1) of the config-3 workload at the reference's grid parameters: "
                      f"{VCM_LIGHT_PATHS} light paths, {VCM_W}x{VCM_H} camera samples; the light pass includes the "
                      f"grid build, the camera pass the merging queries; traversal = the oracle's CPU restatement"}


def run_config1(cpu_threads: int = 0, frames: int = 10):
    """Config 1 (32 displaced icospheres + ground + 2-triangle area light, 512x512, 1 spp,
    4 bounces = max_path_len 5, roulette from bounce 0 as the reference): GPU frame time and
    Mrays/s through PathTracer, beside the reference's PathTracer on all host threads."""
    import torch
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200.integrators import GpuScene, PathTracer
    desc = G.config1(width=512, height=512)
    gs = GpuScene(desc)
    pt = PathTracer(gs, max_path_len=5, rr_start=0)
    image = torch.zeros((512, 512, 3), dtype=torch.float32, device="cuda")
    for k in range(3):
        pt.render(1, 70 + k, image=image)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rays = 0
    e0.record()
    for k in range(frames):
        pt.render(1, 100 + k, image=image)
        rays += int(pt.last_stats[0] + pt.last_stats[1])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / frames
    out = {"workload": f"config 1: {desc.instanced_triangles} triangles, 512x512, 1 spp, max_path_len 5 (4 bounces), "
                       f"roulette from bounce 0", "frame_ms": round(ms, 3),
           "mrays_s": round(rays / frames / (ms * 1e-3) / 1e6, 1), "rays_per_frame": rays // frames}
    pt.close()
    gs.close()
    if cpu_threads:
        from oracle import refwrap as R
        with _StdoutToStderr():
            rs = R.RefScene(desc)
            t0 = time.perf_counter()
            _, a, b = rs.render_pt_threads(512, 512, 1, 5, 100, cpu_threads)
            el = time.perf_counter() - t0
            rs.close()
        out["cpu_baseline"] = {"kind": "reference", "cores": cpu_threads, "cpu_model": cpu_model(),
                               "value": round((a + b) / el / 1e6, 3), "unit": "Mrays/s", "frame_ms": round(el * 1e3, 1),
                               "sample": f"one full frame ({a + b} rays counted by the reference scheduler): the "
                                         f"reference's PathTracer+TileScheduler with the oracle CPU traversal"}
    return out


def N_light_vertices(vi):
    from imbatracer_b200 import native as N
    return max(int(N.load().imbart_vcm_copy_light_vertices(vi.ctx, None, 0)), 0)


def run_serving(scenes=None, config5_rates=(150.0, 400.0), config5_s=3.0, saturation=True):
    """Config 4 (closed batch of 256 renders) and config 5 (Poisson arrivals) in both arms."""
    import torch
    from imbatracer_b200 import scenegen as G
    scenes = scenes or serve_scenes()
    out = {"scenes": len(scenes), "scene_triangles": [d.instanced_triangles for d, _ in scenes],
           "max_path_len": SERVE_MAX_PATH_LEN, "paths_per_wavefront": SERVE_PATHS,
           "pool_bytes": SERVE_BUDGET}
    jobs4 = G.config4_requests()
    mix = {k: sum(1 for j in jobs4 if j.integrator == k) for k in ("pt", "bpt", "vcm")}
    c4 = {"workload": f"{len(jobs4)} renders at once, square, 64^2-1024^2 px log-uniform, spp in {{1,4,16,64}}; "
                      f"integrators {mix['pt']} PT / {mix['bpt']} BPT / {mix['vcm']} VCM (BPT and VCM: spp "
                      f"iterations of one camera sample per pixel and width*height/2 light paths)"}
    for mode in ("plain", "batched"):
        c4[mode] = serve_arm(mode, scenes, jobs4, open_loop=False)
    c4["requests_per_s_ratio"] = round(c4["batched"]["requests_per_s"] / c4["plain"]["requests_per_s"], 3)
    c4["p99_ratio"] = round(c4["plain"]["p99_ms"] / c4["batched"]["p99_ms"], 3)
    out["config4"] = c4
    out["admission"] = admission_times(scenes)
    if config5_rates:
        n_rays = 4 << 20
        ray_buf = torch.empty((n_rays, 8), dtype=torch.float32).pin_memory().numpy()
        r = G.random_rays(np.random.default_rng(5), n_rays, -12.0, 12.0)
        ray_buf[:] = r.view(np.float32).reshape(n_rays, 8)
        hit_buf = torch.empty((n_rays, 4), dtype=torch.int32).pin_memory().numpy()   # shared by all batches
        out["config5"] = []
        for rate in config5_rates:
            jobs5 = G.config5_requests(rate=rate, duration_s=config5_s)
            c5 = {"rate_per_s": rate,
                  "workload": f"Poisson arrivals at {rate:g} req/s for {config5_s:g} s ({len(jobs5)} requests): "
                              f"1920x1080 1-spp increments and ray batches of 64k-4M rays (half each; pinned host "
                              f"buffers)"}
            for mode in ("plain", "batched"):
                c5[mode] = serve_arm(mode, scenes, jobs5, open_loop=True, ray_buf=ray_buf, hit_buf=hit_buf)
            c5["p99_ratio"] = round(c5["plain"]["p99_ms"] / c5["batched"]["p99_ms"], 3)
            out["config5"].append(c5)
        if saturation:
            out["config5_saturation"] = config5_saturation(scenes, ray_buf, hit_buf)
    return out


def config5_saturation(scenes, ray_buf, hit_buf, p99_bound_ms=100.0, duration_s=1.5, start=200.0, step=1.5,
                       top=4000.0, bisections=3):
    """The highest Poisson arrival rate of the config-5 mix each arm sustains: rates grow by
    `step` from `start` while the arm serves at least 95 % of the offered rate with p99
    latency within the bound; then `bisections` geometric midpoints between the last rate that
    passed and the first that failed narrow the bracket. The highest rate that passed is the
    arm's sustained rate."""
    from imbatracer_b200 import scenegen as G
    out = {"p99_bound_ms": p99_bound_ms, "seconds_per_rate": duration_s,
           "rule": "sustained = served >= 0.95 x offered and p99 <= bound"}
    for mode in ("plain", "batched"):
        rate, best, tried, failed = start, None, [], None

        def attempt(rate):
            jobs = G.config5_requests(seed=int(rate), rate=rate, duration_s=duration_s)
            r = serve_arm(mode, scenes, jobs, open_loop=True, ray_buf=ray_buf, hit_buf=hit_buf)
            ok = r["requests_per_s"] >= 0.95 * rate and r["p99_ms"] <= p99_bound_ms
            tried.append({"rate": round(rate, 1), "served": r["requests_per_s"], "p99_ms": r["p99_ms"],
                          "p50_ms": r["p50_ms"], "sustained": ok})
            return r, ok

        while rate <= top:
            r, ok = attempt(rate)
            if not ok:
                failed = rate
                break
            best = r | {"rate": round(rate, 1)}
            rate *= step
        lo = best["rate"] if best else None
        for _ in range(bisections if (lo and failed) else 0):
            mid = (lo * failed) ** 0.5
            r, ok = attempt(mid)
            if ok:
                best, lo = r | {"rate": round(mid, 1)}, mid
            else:
                failed = mid
        out[mode] = {"sustained_rate_per_s": best["rate"] if best else None,
                     "requests_per_s": best["requests_per_s"] if best else None,
                     "p99_ms": best["p99_ms"] if best else None, "sweep": tried}
    if out["plain"]["requests_per_s"] and out["batched"]["requests_per_s"]:
        out["requests_per_s_ratio"] = round(out["batched"]["requests_per_s"] / out["plain"]["requests_per_s"], 3)
    return out


# ---------------------------------------------------------------------------------------
# --mode trace: traversal kernels alone on fixed ray sets of the frame (kernel tuning)
# ---------------------------------------------------------------------------------------
def make_scene(name: str = "config2"):
    from imbatracer_b200 import scene as S
    from imbatracer_b200 import scenegen as G
    desc = {"config1": G.config1, "config2": G.config2, "config3": G.config3}[name]()
    td = S.build_traversal_data(desc.meshes, desc.instances)
    return desc, td


def make_wavefront(desc, ds, torch, dev, seed: int, shadow_from_bounce: bool = False):
    """Primary camera rays, one bounce of incoherent secondary rays from their hits, and one
    shadow ray per hit towards a random light point (untimed set-up on the device). With
    shadow_from_bounce the shadow set also holds one shadow ray per hit of the secondary rays
    and the secondary set a second bounce from those hits (as in a frame, where most rays
    start at bounce hits)."""
    cam = desc.camera
    w, h = cam.width, cam.height
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    pos = torch.tensor(cam.pos, dtype=torch.float32, device=dev)
    fwd = torch.tensor(cam.dir, dtype=torch.float32, device=dev)
    fwd = fwd / fwd.norm()
    up = torch.tensor(cam.up, dtype=torch.float32, device=dev)
    right = torch.linalg.cross(fwd, up)
    right = right / right.norm()
    upv = torch.linalg.cross(right, fwd)
    scale = float(np.tan(np.radians(cam.fov) / 2)) * 2.0 / h
    ys, xs = torch.meshgrid(torch.arange(h, device=dev), torch.arange(w, device=dev), indexing="ij")
    px = (xs.float() + torch.rand((h, w), generator=g, device=dev) - w / 2) * scale
    py = (h / 2 - ys.float() - torch.rand((h, w), generator=g, device=dev)) * scale
    d = fwd + px[..., None] * right + py[..., None] * upv
    d = (d / d.norm(dim=-1, keepdim=True)).reshape(-1, 3)
    n = d.shape[0]
    prim = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    prim[:, :3] = pos
    prim[:, 4:7] = d
    prim[:, 7] = 3.0e38
    hits = torch.zeros((n, 4), dtype=torch.int32, device=dev)
    ds.trace(prim, hits)
    torch.cuda.synchronize()
    hit = hits[:, 0] >= 0
    t = hits[:, 2].view(torch.float32)
    p = prim[:, :3] + t[:, None] * prim[:, 4:7]
    hp, hd, ht = p[hit], prim[hit, 4:7], t[hit]
    m = hp.shape[0]
    sd = torch.randn((m, 3), generator=g, device=dev)
    sd = sd / sd.norm(dim=-1, keepdim=True)
    flip = (sd * hd).sum(-1) > 0
    sd[flip] = -sd[flip]
    sec = torch.zeros((m, 8), dtype=torch.float32, device=dev)
    sec[:, :3] = hp
    sec[:, 3] = 1e-3 * ht
    sec[:, 4:7] = sd
    sec[:, 7] = 3.0e38
    lights = torch.tensor(np.stack([np.stack(l[:3]) for l in desc.lights]), dtype=torch.float32, device=dev)
    li = torch.randint(0, lights.shape[0], (m,), generator=g, device=dev)
    r1 = torch.rand(m, generator=g, device=dev).sqrt()
    r2 = torch.rand(m, generator=g, device=dev)
    bu, bv = 1 - r1, r2 * r1
    tri = lights[li]
    lp = bu[:, None] * tri[:, 0] + bv[:, None] * tri[:, 1] + (1 - bu - bv)[:, None] * tri[:, 2]
    dv = lp - hp
    dist = dv.norm(dim=-1)
    off = 1e-3 * dist
    sh = torch.zeros((m, 8), dtype=torch.float32, device=dev)
    sh[:, :3] = hp
    sh[:, 3] = off
    sh[:, 4:7] = dv / dist[:, None]
    sh[:, 7] = dist - off
    if shadow_from_bounce:
        shits = torch.zeros((m, 4), dtype=torch.int32, device=dev)
        ds.trace(sec.contiguous(), shits)
        torch.cuda.synchronize()
        sh2 = shadow_rays_from(sec, shits, lights, g, torch, dev)
        sh = torch.cat([sh, sh2], 0)
        # A second bounce: uniform directions in the hemisphere facing back along each hit ray.
        hit2 = shits[:, 0] >= 0
        t2 = shits[:, 2].view(torch.float32)
        p2 = (sec[:, :3] + t2[:, None] * sec[:, 4:7])[hit2]
        d2 = sec[hit2, 4:7]
        k = p2.shape[0]
        nd = torch.randn((k, 3), generator=g, device=dev)
        nd = nd / nd.norm(dim=-1, keepdim=True)
        flip2 = (nd * d2).sum(-1) > 0
        nd[flip2] = -nd[flip2]
        ter = torch.zeros((k, 8), dtype=torch.float32, device=dev)
        ter[:, :3] = p2
        ter[:, 3] = 1e-3 * t2[hit2]
        ter[:, 4:7] = nd
        ter[:, 7] = 3.0e38
        sec = torch.cat([sec, ter], 0)
    return [(prim.contiguous(), False), (sec.contiguous(), False), (sh.contiguous(), True)]


def shadow_rays_from(rays, hits, lights, g, torch, dev):
    """One shadow ray per hit of `rays` towards a random point of a random light triangle."""
    hit = hits[:, 0] >= 0
    t = hits[:, 2].view(torch.float32)
    p = (rays[:, :3] + t[:, None] * rays[:, 4:7])[hit]
    m = p.shape[0]
    li = torch.randint(0, lights.shape[0], (m,), generator=g, device=dev)
    r1 = torch.rand(m, generator=g, device=dev).sqrt()
    r2 = torch.rand(m, generator=g, device=dev)
    bu, bv = 1 - r1, r2 * r1
    tri = lights[li]
    lp = bu[:, None] * tri[:, 0] + bv[:, None] * tri[:, 1] + (1 - bu - bv)[:, None] * tri[:, 2]
    dv = lp - p
    dist = dv.norm(dim=-1)
    off = 1e-3 * dist
    out = torch.zeros((m, 8), dtype=torch.float32, device=dev)
    out[:, :3] = p
    out[:, 3] = off
    out[:, 4:7] = dv / dist[:, None]
    out[:, 7] = dist - off
    return out


def run_trace(args):
    import torch
    from imbatracer_b200 import native as N
    from imbatracer_b200 import scene as S
    dev = torch.device("cuda", 0)
    desc, td = make_scene(args.scene)
    ds = S.DeviceScene(td)
    sets = make_wavefront(desc, ds, torch, dev, 1234)
    hits = [torch.zeros((r.shape[0], 4), dtype=torch.int32, device=dev) for r, _ in sets]
    for _ in range(args.warmup):
        for (r, a), h in zip(sets, hits):
            ds.trace(r, h, any_hit=a)
    torch.cuda.synchronize()
    out = {}
    for name, (r, a), h in zip(["primary", "secondary", "shadow"], sets, hits):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            ds.trace(r, h, any_hit=a)
        e1.record()
        torch.cuda.synchronize()
        out[name] = round(r.shape[0] * args.steps / (e0.elapsed_time(e1) * 1e-3) / 1e6, 1)
    print(json.dumps({"mode": "trace", "scene": args.scene, "Mrays_s": out, "rays": [r.shape[0] for r, _ in sets]}),
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="pt", choices=["pt", "trace", "serve", "vcm"])
    ap.add_argument("--scene", default="config2", choices=["config1", "config2", "config3"],
                    help="trace mode: the scene whose frame's ray sets are traced")
    ap.add_argument("--no-vcm", action="store_true", help="pt mode: skip the VCM-family iterations")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="pt mode: keep the default kernel configurations")
    ap.add_argument("--paths-in-flight", type=int, default=0,
                    help="pt mode: wavefront size (paths in flight) instead of the autotuner's pick")
    ap.add_argument("--no-serving", action="store_true", help="pt mode: skip the serving comparison")
    ap.add_argument("--no-config3", action="store_true", help="pt mode: skip the config-3 traversal roofline")
    ap.add_argument("--no-config1", action="store_true", help="pt mode: skip the config-1 frame and its CPU baseline")
    ap.add_argument("--rate", type=float, nargs="*", default=[150.0, 400.0],
                    help="serve mode: config 5 arrival rates (req/s)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.warmup < 3:
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3
    if args.mode == "trace":
        run_trace(args)
    elif args.mode == "vcm":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"mode": "vcm", "vcm_family": run_vcm(args.steps, args.warmup),
                              "config3_spec": run_vcm_spec()}), flush=True)
    elif args.mode == "serve":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"mode": "serve", "serving": run_serving(config5_rates=tuple(args.rate))}), flush=True)
    else:
        run_pt(args)


if __name__ == "__main__":
    main()
