"""Multi-rank paths: the bench's whole-job timing (max time, summed units over ranks) and the
multi-GPU VCM iteration (light-path ranges, all-gather of light vertices back into the
single-GPU cache order, camera-sample ranges, summed images).

CPU: two gloo ranks (processes) run the collectives on CPU tensors. GPU (one device): the
ranks of a multi-GPU iteration are emulated one after another on the same GPU, with the
same assembly code, and must reproduce the single-GPU cache bit for bit and its image up
to float summation order; a one-rank NCCL group runs the distributed integrator itself.
"""
import os
import socket

import numpy as np
import pytest

from imbatracer_b200 import distributed as D


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_split_range_covers_every_item_once():
    for total in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            got = [D.split_range(total, r, world) for r in range(world)]
            assert got[0][0] == 0
            for (f0, n0), (f1, _) in zip(got, got[1:]):
                assert f0 + n0 == f1
            assert sum(n for _, n in got) == total
            assert max(n for _, n in got) - min(n for _, n in got) <= 1


def fake_cache(rank, waves):
    """Vertices tagged (rank, wavefront, index in wavefront) in their first three floats."""
    import torch
    rows = []
    for w, c in enumerate(waves):
        for i in range(c):
            rows.append([rank, w, i] + [0.25 * rank] * 25)
    return torch.tensor(rows, dtype=torch.float32).reshape(-1, 28)


WAVES = {0: [3, 0, 2, 1], 1: [1, 4, 0, 0]}


def _gloo_worker(rank, world, port, result_dir):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, units = bench.job_totals(10.0 + rank, 100 * (rank + 1), torch.device("cpu"), world)
        assert ms == 10.0 + world - 1 and units == sum(100 * (r + 1) for r in range(world))
        g = D.all_gather_light_vertices(fake_cache(rank, WAVES[rank]), WAVES[rank])
        tags = [tuple(int(x) for x in row[:3]) for row in g.tolist()]
        expect = [(r, w, i) for w in range(4) for r in range(world) for i in range(WAVES[r][w])]
        assert tags == expect, (tags, expect)
        # A rank with an empty range and no vertices.
        waves = [0, 0, 0, 0] if rank == 1 else WAVES[0]
        g = D.all_gather_light_vertices(fake_cache(rank, waves), waves)
        assert [tuple(int(x) for x in row[:3]) for row in g.tolist()] == \
            [(0, w, i) for w in range(4) for i in range(WAVES[0][w])]
        # A frame split by sample ranges: every sample lands once in the summed image.
        pt = FakePathTracer()
        img = D.render_frame_split(pt, 3, 7, device="cpu")
        assert torch.equal(img, FakePathTracer.whole(3)), img
        assert pt.ranges[0][0] == (0 if rank == 0 else pt.ranges[0][0]) and len(pt.ranges) == 1
        open(os.path.join(result_dir, f"ok{rank}"), "w").write("ok")
    finally:
        dist.destroy_process_group()


class FakePathTracer:
    """Stands in for PathTracer on the CPU: render() adds 1 + sample index to the sample's
    pixel (sample index // spp) for every sample of its range."""

    class scene:
        class desc:
            class camera:
                width, height = 5, 4

    def __init__(self):
        self.ranges = []

    def render(self, spp, seed_base, w, h, image=None, stream=None, sample_range=None):
        first, count = sample_range
        self.ranges.append((first, count))
        for i in range(first, first + count):
            image.view(-1, 3)[i // spp] += 1.0 + i
        self.last_stats = np.zeros(3, np.int64)
        return image

    @staticmethod
    def whole(spp):
        import torch
        img = torch.zeros((4, 5, 3), dtype=torch.float32)
        for i in range(4 * 5 * spp):
            img.view(-1, 3)[i // spp] += 1.0 + i
        return img


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_gloo_worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert os.path.exists(tmp_path / "ok0") and os.path.exists(tmp_path / "ok1")


def test_assembly_rejects_inconsistent_counts():
    import torch
    with pytest.raises(ValueError):
        D.assemble_light_vertices([torch.zeros((3, 28))], [[1, 1]])


@pytest.mark.gpu
@pytest.mark.parametrize("algo,ranks", [("vcm", 2), ("bpt", 3), ("ppm", 2)])
def test_emulated_ranks_reproduce_the_single_gpu_iteration(cuda, algo, ranks):
    import torch
    from imbatracer_b200.integrators import GpuScene, VcmIntegrator
    from tests.test_pt import small_mixed_scene
    d = small_mixed_scene()
    gs = GpuScene(d)
    w, h, kw = 48, 32, dict(max_path_len=6, light_path_count=1500)
    one = VcmIntegrator(gs, algo, w, h, **kw)
    one.begin_iteration(2)
    ref = one.light_pass(71, 5)
    ref_cache = one.light_vertices()
    ref = one.camera_pass(72, image=ref).cpu().numpy()
    parts, waves, imgs, ctxs = [], [], [], []
    for r in range(ranks):
        vi = VcmIntegrator(gs, algo, w, h, **kw)
        vi.begin_iteration(2)
        first, n = D.split_range(1500, r, ranks)
        img, wv = vi.light_pass_range(first, n, 71, 5)
        parts.append(vi.light_vertices_device())
        waves.append(wv.tolist())
        imgs.append(img)
        ctxs.append(vi)
    glob = D.assemble_light_vertices(parts, waves)
    assert np.array_equal(glob.cpu().numpy().view(np.int32), ref_cache.view(np.int32))
    total = w * h
    for r, vi in enumerate(ctxs):
        vi.load_light_vertices(glob)
        c0, cn = D.split_range(total, r, ranks)
        vi.camera_pass_range(c0, cn, 72, image=imgs[r])
    summed = sum(i.cpu().numpy().astype(np.float64) for i in imgs)
    den = np.sqrt(np.mean(ref.astype(np.float64) ** 2))
    assert ref.sum() > 0 and np.sqrt(np.mean((summed - ref) ** 2)) / den <= 1e-5
    for vi in ctxs:
        vi.close()
    one.close()


@pytest.mark.gpu
def test_distributed_integrator_on_one_nccl_rank(cuda):
    import torch
    import torch.distributed as dist
    from imbatracer_b200.integrators import GpuScene, VcmIntegrator
    from tests.test_pt import small_mixed_scene
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        d = small_mixed_scene()
        gs = GpuScene(d)
        kw = dict(max_path_len=6, light_path_count=1200)
        dv = D.DistributedVcmIntegrator(gs, "vcm", 40, 24, **kw)
        vi = VcmIntegrator(gs, "vcm", 40, 24, **kw)
        a = None
        b = None
        for it in (1, 2):
            a = dv.render(it, 300 + it, 400 + it, 9, image=a)
            b = vi.render(it, 300 + it, 400 + it, 9, image=b)
        a, b = a.cpu().numpy(), b.cpu().numpy()
        den = np.sqrt(np.mean(b.astype(np.float64) ** 2))
        assert b.sum() > 0 and np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / den <= 1e-5
        dv.close()
        vi.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("ranks,graphs,paths", [(2, 2, 0), (3, 2, 5000), (3, 0, 0)])
def test_frame_split_by_sample_ranges_equals_the_frame(cuda, ranks, graphs, paths):
    """A path-traced frame split into `ranks` contiguous sample ranges (emulated ranks rendered
    one after another on this GPU, as render_frame_split does on each rank) sums to the
    single-GPU frame up to float summation order, with the same closest-hit and shadow ray
    counts; with the bounce loop as CUDA graphs (2) and driven from the host (0), and with a
    wavefront smaller than a range (several ranges per rank)."""
    import torch
    from imbatracer_b200 import native as N
    from imbatracer_b200.integrators import GpuScene, PathTracer
    from tests.test_pt import small_mixed_scene
    d = small_mixed_scene()
    gs = GpuScene(d)
    pt = PathTracer(gs, max_path_len=6)
    if paths:
        pt.max_paths = paths
    N.check(N.load().imbart_pt_set_graphs(pt.ctx, graphs), "imbart_pt_set_graphs")
    w, h, spp = 48, 32, 4
    whole = pt.render(spp, 21, w, h)
    whole_stats = pt.last_stats.copy()
    split = torch.zeros_like(whole)
    stats = np.zeros(3, np.int64)
    for r in range(ranks):
        first, count = D.split_range(w * h * spp, r, ranks)
        pt.render(spp, 21, w, h, image=split, sample_range=(first, count))
        stats += pt.last_stats
    torch.cuda.synchronize()
    a, b = split.cpu().numpy().astype(np.float64), whole.cpu().numpy().astype(np.float64)
    assert b.sum() > 0
    assert np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)) <= 1e-6
    assert stats[0] == whole_stats[0] and stats[1] == whole_stats[1]
    with pytest.raises(N.ImbartError):
        pt.render(spp, 21, w, h, sample_range=(w * h * spp - 10, 11))   # past the frame's samples
    N.load().imbart_clear_error()
    pt.close()
    gs.close()


@pytest.mark.gpu
def test_render_frame_split_on_one_nccl_rank(cuda):
    import torch
    import torch.distributed as dist
    from imbatracer_b200.integrators import GpuScene, PathTracer
    from tests.test_pt import small_mixed_scene
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        gs = GpuScene(small_mixed_scene())
        pt = PathTracer(gs, max_path_len=6)
        a = D.render_frame_split(pt, 2, 33, 40, 24)
        b = pt.render(2, 33, 40, 24)
        torch.cuda.synchronize()
        a, b = a.cpu().numpy().astype(np.float64), b.cpu().numpy().astype(np.float64)
        assert b.sum() > 0 and np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)) <= 1e-6
        pt.close()
        gs.close()
    finally:
        dist.destroy_process_group()
