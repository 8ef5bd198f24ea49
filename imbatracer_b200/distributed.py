"""VCM-family iterations on several GPUs (one process per GPU, torch.distributed).

The reference renders an iteration on one machine (VCMIntegrator::render, vcm.cpp:25-55):
trace the light paths and store their vertices, build the photon grid over them, trace the
camera paths against them. Across G ranks:

  1. each rank traces a contiguous range of the iteration's light paths (paths are seeded by
     their global index, so the ranges together are exactly the single-GPU paths);
  2. the ranks' light vertices are all-gathered (NCCL over NVLink; one variable-size
     exchange per iteration) and put back into the single-GPU order, wavefront by wavefront
     and within a wavefront by rank: every rank then holds the same cache as one GPU would,
     and builds the photon grid over it;
  3. each rank traces a contiguous range of the camera samples against that cache;
  4. the ranks' images of the iteration (their light-tracing splats and their camera
     samples) are summed with an all-reduce.

The image equals the single-GPU iteration's up to the order of the float additions. PT
frames and ray batches need no exchange (the bench runs them as independent replicas); one
PT frame can also be split across the ranks by sample ranges (render_frame_split: samples
are seeded by their index, so the ranges' images summed are the single-GPU frame).
"""
from __future__ import annotations

import numpy as np

from .integrators import GpuScene, VcmIntegrator


def split_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """(first, count) of rank's contiguous share of [0, total): the first total % world
    ranks take one more."""
    base, extra = divmod(int(total), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def assemble_light_vertices(parts, wave_counts):
    """Single-GPU cache order from per-rank caches: parts[r] is rank r's (n_r, 28) cache in
    (wavefront, path) order, wave_counts[r][w] the vertices its wavefront w added. The result
    lists wavefront 0 of every rank (in rank order), then wavefront 1, and so on."""
    import torch
    segs = []
    offs = [0] * len(parts)
    n_waves = max(len(w) for w in wave_counts)
    for w in range(n_waves):
        for r, p in enumerate(parts):
            c = int(wave_counts[r][w]) if w < len(wave_counts[r]) else 0
            if c:
                segs.append(p[offs[r]:offs[r] + c])
                offs[r] += c
    for r, p in enumerate(parts):
        if offs[r] != p.shape[0]:
            raise ValueError("light vertex counts do not add up")
    if not segs:
        return parts[0][:0]
    return torch.cat(segs, 0)


def all_gather_light_vertices(local, wave_counts, group=None):
    """All ranks' caches in the single-GPU order (see assemble_light_vertices); local: this
    rank's (n, 28) float32 tensor, wave_counts: its per-wavefront counts (same length on
    every rank). Works for CUDA tensors over NCCL and CPU tensors over gloo."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = local.device
    waves = torch.as_tensor(np.asarray(wave_counts, np.int64), device=dev)
    all_waves = [torch.zeros_like(waves) for _ in range(world)]
    dist.all_gather(all_waves, waves, group=group)
    counts = [int(w.sum().item()) for w in all_waves]
    if counts[dist.get_rank(group)] != local.shape[0]:
        raise ValueError("the local cache does not match its wavefront counts")
    cap = max(max(counts), 1)
    padded = torch.zeros((cap, 28), dtype=local.dtype, device=dev)
    padded[:local.shape[0]] = local
    gathered = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(gathered, padded, group=group)
    parts = [gathered[r][:counts[r]] for r in range(world)]
    return assemble_light_vertices(parts, [w.tolist() for w in all_waves])


def render_frame_split(pt, spp: int, seed_base: int, width: int | None = None, height: int | None = None,
                       image=None, group=None, stream=None, device=None):
    """One path-traced frame split across the ranks of `group`: rank r renders its contiguous
    share of the frame's width * height * spp samples (PathTracer.render with sample_range)
    and the ranks' images are summed with an all-reduce, so every rank gets the whole frame —
    the single-GPU image up to the order of the float additions. Returns the summed image
    (added to `image` when given); pt.last_stats holds this rank's ray counts. device: where
    the image lives (default: the path tracer's GPU)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    cam = pt.scene.desc.camera
    w, h = width or cam.width, height or cam.height
    dev = torch.device(device) if device is not None else torch.device("cuda", pt.scene.device)
    part = torch.zeros((h, w, 3), dtype=torch.float32, device=dev)
    first, count = split_range(w * h * spp, rank, world)
    if count > 0:
        pt.render(spp, seed_base, w, h, image=part, stream=stream, sample_range=(first, count))
    else:
        pt.last_stats = np.zeros(3, np.int64)
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    dist.all_reduce(part, group=group)
    if image is None:
        return part
    image += part
    return image


class DistributedVcmIntegrator:
    """VcmIntegrator over the ranks of a torch.distributed group: every rank calls render()
    with the same arguments and gets the same summed image."""

    def __init__(self, scene: GpuScene, algorithm: str = "vcm", width: int | None = None, height: int | None = None,
                 group=None, **settings):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.vi = VcmIntegrator(scene, algorithm, width, height, **settings)

    def render(self, iteration: int, light_seed: int, camera_seed: int, light_seed_step: int = 0, image=None):
        import torch
        import torch.distributed as dist
        vi = self.vi
        part = torch.zeros((vi.height, vi.width, 3), dtype=torch.float32,
                           device=torch.device("cuda", vi.scene.device))
        vi.begin_iteration(iteration)
        first, n = split_range(vi.settings.light_path_count, self.rank, self.world)
        _, waves = vi.light_pass_range(first, n, light_seed, light_seed_step, image=part)
        local = vi.light_vertices_device()
        vi.load_light_vertices(all_gather_light_vertices(local, waves, self.group))
        total = vi.width * vi.height * vi.settings.spp
        c0, cn = split_range(total, self.rank, self.world)
        vi.camera_pass_range(c0, cn, camera_seed, image=part)
        torch.cuda.synchronize()
        dist.all_reduce(part, group=self.group)
        if image is None:
            return part
        image += part
        return image

    def close(self):
        self.vi.close()
