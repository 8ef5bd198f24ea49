"""Benchmark of the wavefront hot path (Mrays/s, closest + shadow rays).

Workload: the 1920x1080 instanced scene (200 instances of 8 seeded meshes, ~1.14M instanced
triangles, 16 area lights + environment). One step traces one wavefront of that frame's rays
through libimbart: the primary camera rays (closest hit), one bounce of incoherent secondary
rays from the primary hits (closest hit) and one shadow ray per primary hit towards a random
point on a random area light (any hit). Inputs are resident in HBM when timing starts; the
rays and hits of one step (~300 MB) exceed the 126 MB L2.

`value` is device-timed Mrays/s over all ranks; `e2e` is the same metric through the host
buffer C-ABI entry (pinned host rays copied in, hits copied out inside the timed region).
`--impl reference` times the CPU traversal (the oracle restatement of the reference's
traversal boundary; the reference's own traversal library is not in its tree) on all host
cores on a bounded sample of the same rays.
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

WORKLOAD = "wavefront_1080p_instanced_200x8"
METRIC = "Mrays/s closest+shadow"


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
        # Wait for the first sample so that the timed region is covered.
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def mark(self):
        """Starts counting samples from here (the timed region)."""
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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # Samples from the timed region; keep the one before it when the region is shorter
        # than the sampling interval.
        lines = self.lines[max(getattr(self, "first", 0) - 1, 0):]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene():
    from imbatracer_b200 import scenegen as G
    from imbatracer_b200 import scene as S
    desc = G.config2()
    td = S.build_traversal_data(desc.meshes, desc.instances)
    return desc, td


def make_wavefront(desc, ds, torch, dev, seed: int):
    """Builds the step's three ray sets on the device (untimed setup)."""
    from imbatracer_b200 import native as N
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
    jx = torch.rand((h, w), generator=g, device=dev)
    jy = torch.rand((h, w), generator=g, device=dev)
    px = (xs.float() + jx - w / 2) * scale
    py = (h / 2 - ys.float() - jy) * scale
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
    # Secondary rays: uniform directions on the hemisphere facing back along the ray.
    sd = torch.randn((m, 3), generator=g, device=dev)
    sd = sd / sd.norm(dim=-1, keepdim=True)
    flip = (sd * hd).sum(-1) > 0
    sd[flip] = -sd[flip]
    sec = torch.zeros((m, 8), dtype=torch.float32, device=dev)
    sec[:, :3] = hp
    sec[:, 3] = 1e-3 * ht
    sec[:, 4:7] = sd
    sec[:, 7] = 3.0e38
    # Shadow rays towards a random point on a random light (offset as pt.cpp:37-41).
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
    return [(prim.contiguous(), False), (sec.contiguous(), False), (sh.contiguous(), True)]


def algorithmic_bytes(ds, sets, torch, dev):
    """Bytes per launch from the statistics variant: 32 B ray + 16 B hit per ray, 80 B per
    8-wide node, 48 B per triangle, 64 B per instance entered."""
    from imbatracer_b200 import native as N
    lib = N.load()
    out = []
    for rays, any_hit in sets:
        st = torch.zeros(3, dtype=torch.int64, device=dev)
        hits = torch.zeros((rays.shape[0], 4), dtype=torch.int32, device=dev)
        N.check(lib.imbart_trace_stats(ds.handle, N.ptr(rays), N.ptr(hits), rays.shape[0],
                                       N.TRACE_ANY if any_hit else N.TRACE_CLOSEST, N.ptr(st), None), "stats")
        torch.cuda.synchronize()
        nodes, tris, insts = (int(x) for x in st.cpu())
        out.append({"rays": int(rays.shape[0]), "nodes": nodes, "tris": tris, "insts": insts,
                    "bytes": 48 * int(rays.shape[0]) + 80 * nodes + 48 * tris + 64 * insts})
    return out


def cpu_baseline(td, sets, torch, sample: int, threads: int, seconds: float = 12.0):
    """Times the oracle's traversal on the host cores on a bounded sample of every ray set."""
    from oracle import oracle as O
    from imbatracer_b200 import native as N
    samples = []
    for rays, any_hit in sets:
        r = rays[:sample].cpu().numpy().copy().view(N.RAY_DTYPE).reshape(-1)
        samples.append((np.ascontiguousarray(r), any_hit))
    O.trace_node2(td, samples[0][0][:1000], nthreads=threads)  # warm up
    total, elapsed, reps = 0, 0.0, 0
    while elapsed < seconds or reps == 0:
        t0 = time.perf_counter()
        for r, any_hit in samples:
            O.trace_node2(td, r, any_hit=any_hit, nthreads=threads)
            total += len(r)
        elapsed += time.perf_counter() - t0
        reps += 1
    return total / elapsed / 1e6, total, reps


def run_ours(args):
    import torch
    import torch.distributed as dist
    from imbatracer_b200 import native as N
    from imbatracer_b200 import scene as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = N.load()

    desc, td = make_scene()
    ds = S.DeviceScene(td, device=local)
    sets = make_wavefront(desc, ds, torch, dev, seed=1234 + rank)
    n_rays = sum(r.shape[0] for r, _ in sets)
    hits = [torch.zeros((r.shape[0], 4), dtype=torch.int32, device=dev) for r, _ in sets]
    stream = torch.cuda.current_stream(dev)

    def step(events=None):
        for i, ((rays, any_hit), h) in enumerate(zip(sets, hits)):
            if events is not None:
                events[i][0].record(stream)
            ds.trace(rays, h, any_hit=any_hit, stream=stream)
            if events is not None:
                events[i][1].record(stream)

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches_before = lib.imbart_kernel_launch_count()
    per_launch = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in sets] for _ in range(args.steps)]
    clocks.mark()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        step(per_launch[k])
    end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = lib.imbart_kernel_launch_count() - launches_before
    ms = start.elapsed_time(end)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    launch_ms = np.array([[a.elapsed_time(b) for a, b in row] for row in per_launch]).mean(0)

    # e2e: same metric through the host-buffer entry, pinned host memory, copies inside.
    host_sets = [(r.cpu().pin_memory(), a) for r, a in sets]
    host_hits = [torch.zeros((r.shape[0], 4), dtype=torch.int32).pin_memory() for r, _ in host_sets]

    def e2e_step():
        for (r, a), h in zip(host_sets, host_hits):
            N.check(lib.imbart_trace_host(ds.handle, N.ptr(r), N.ptr(h), r.shape[0],
                                          N.TRACE_ANY if a else N.TRACE_CLOSEST, stream.cuda_stream), "e2e")

    for _ in range(args.warmup):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e_end.record(stream)
    torch.cuda.synchronize()
    e_ms = e_start.elapsed_time(e_end)
    te = torch.tensor([e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e_ms_max = float(te.item())

    stats = algorithmic_bytes(ds, sets, torch, dev)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak_gbs = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = int(np.argmax(launch_ms))
    achieved = stats[dom]["bytes"] / (launch_ms[dom] * 1e-3) / 1e9

    if rank == 0:
        total_rays = n_rays * world * args.steps
        value = total_rays / (ms_max * 1e-3) / 1e6
        e2e_value = total_rays / (e_ms_max * 1e-3) / 1e6
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sample = 65536
            mr, tot, reps = cpu_baseline(td, sets, torch, sample, threads)
            cpu = {"value": round(mr, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                   "sample": f"first {sample} rays of each of the 3 ray sets ({tot} rays over {reps} passes), "
                             f"oracle traversal of the reference layout, {threads} threads"}
        names = ["primary_closest", "secondary_closest", "shadow_any"]
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator; seeded ray sets)",
            "config": {"workload": WORKLOAD, "resolution": "1920x1080", "instances": len(desc.instances),
                       "meshes": len(desc.meshes) - 1, "instanced_triangles": desc.instanced_triangles,
                       "rays_per_step": n_rays, "ray_sets": {nm: s["rays"] for nm, s in zip(names, stats)},
                       "l2": "inputs larger than L2 (rays+hits per step ~%d MB)" % (n_rays * 48 // 2 ** 20),
                       "parallelism": f"replicas x{world} (independent ray wavefronts per GPU)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak_gbs, "unit": "GB/s",
                         "frac": round(achieved / peak_gbs, 4), "traffic": None,
                         "kernel": f"trace_kernel ({names[dom]})", "peak_source": peak_src,
                         "bytes_per_launch": stats[dom]["bytes"], "launch_ms": round(float(launch_ms[dom]), 4),
                         "bytes_per_ray": round(stats[dom]["bytes"] / stats[dom]["rays"], 1)},
            "launch_ms": {nm: round(float(x), 4) for nm, x in zip(names, launch_ms)},
            "work": {nm: {k: s[k] for k in ("nodes", "tris", "insts")} for nm, s in zip(names, stats)},
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": 32 * n_rays, "d2h_bytes_per_step": 16 * n_rays},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """CPU arm: the traversal restatement on all host cores, bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    from imbatracer_b200 import native as N
    from oracle import oracle as O
    desc, td = make_scene()
    # The same three ray sets, built on the CPU from the same generator as the GPU arm would
    # need a GPU; here a bounded sample with the same composition: camera rays, secondary
    # rays and shadow rays traced by the CPU traversal.
    rng = np.random.default_rng(1234)
    cam = desc.camera
    n = 65536
    fwd = np.array(cam.dir, np.float64); fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, cam.up); right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    scale = np.tan(np.radians(cam.fov) / 2) * 2.0 / cam.height
    pix = rng.integers(0, cam.width * cam.height, n)
    px = (pix % cam.width + rng.random(n) - cam.width / 2) * scale
    py = (cam.height / 2 - pix // cam.width - rng.random(n)) * scale
    d = fwd + px[:, None] * right + py[:, None] * upv
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    prim = np.zeros(n, N.RAY_DTYPE)
    prim["org"][:, :3] = cam.pos
    prim["dir"][:, :3] = d
    prim["dir"][:, 3] = 3e38
    threads = os.cpu_count() or 1
    h = O.trace_node2(td, prim, nthreads=threads)
    hit = h["tri_id"] >= 0
    hp = (prim["org"][hit, :3] + h["tmax"][hit, None] * prim["dir"][hit, :3]).astype(np.float32)
    m = len(hp)
    sd = rng.normal(size=(m, 3)); sd /= np.linalg.norm(sd, axis=1, keepdims=True)
    flip = (sd * prim["dir"][hit, :3]).sum(1) > 0
    sd[flip] *= -1
    sec = np.zeros(m, N.RAY_DTYPE)
    sec["org"][:, :3] = hp
    sec["org"][:, 3] = 1e-3 * h["tmax"][hit]
    sec["dir"][:, :3] = sd
    sec["dir"][:, 3] = 3e38
    lights = np.stack([np.stack(l[:3]) for l in desc.lights])
    li = rng.integers(0, len(lights), m)
    r1 = np.sqrt(rng.random(m)); r2 = rng.random(m)
    bu, bv = 1 - r1, r2 * r1
    lp = bu[:, None] * lights[li, 0] + bv[:, None] * lights[li, 1] + (1 - bu - bv)[:, None] * lights[li, 2]
    dv = lp - hp
    dist = np.linalg.norm(dv, axis=1)
    sh = np.zeros(m, N.RAY_DTYPE)
    sh["org"][:, :3] = hp
    sh["org"][:, 3] = 1e-3 * dist
    sh["dir"][:, :3] = dv / dist[:, None]
    sh["dir"][:, 3] = dist - 1e-3 * dist
    sets = [(prim, False), (sec, False), (sh, True)]
    for _ in range(args.warmup):
        for r, a in sets:
            O.trace_node2(td, r[:4096], any_hit=a, nthreads=threads)
    total, t0 = 0, time.perf_counter()
    for _ in range(args.steps):
        for r, a in sets:
            O.trace_node2(td, r, any_hit=a, nthreads=threads)
            total += len(r)
    el = time.perf_counter() - t0
    value = total / el / 1e6
    line = {"metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "impl": "reference",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(el / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator; seeded ray sets)",
            "config": {"workload": WORKLOAD, "rays_per_step": total // args.steps,
                       "sample": "65536 camera rays + their secondary and shadow rays per step"},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"{total // args.steps} rays per step (65536 camera rays + secondary + shadow)"},
            "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
