"""Sample generation and the wavefront path tracer against the reference itself.

Camera rays and RNG states must equal the reference's PixelRayGen + PerspectiveCamera bit
for bit. Images from identical per-pixel seeding must be within relative RMSE 1e-3 of the
reference's PathTracer (the reference's own pt.cpp, built in oracle/_ref, tracing through
the oracle traversal) at the same spp: paths are deterministic per sample, so the only
differences are float rounding in transcendental functions and atomic accumulation order,
which can flip a rare Russian-roulette or lobe decision.
"""
import numpy as np
import pytest

from imbatracer_b200 import native as N
from imbatracer_b200 import scenegen as G
from oracle import refwrap as R
from tests import helpers as H

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference tree absent)")

RMSE_TOL = 1e-3


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / np.sqrt(np.mean(b.astype(np.float64) ** 2)))


def small_mixed_scene():
    """Every material kind, a constant environment and triangle lights, instanced meshes."""
    rng = np.random.default_rng(5)
    meshes, materials, instances = [], [], []
    kinds = [G.LAMBERT, G.PHONG, G.GLOSSY, G.MIRROR, G.GLASS]
    for k, kind in enumerate(kinds):
        v, f = G.displaced_sphere(rng, 2, (0, 0, 0), 1.0)
        if kind == G.LAMBERT:
            mat = G.Material(G.LAMBERT, color=(0.7, 0.5, 0.3))
        elif kind == G.PHONG:
            mat = G.Material(G.PHONG, color=(0.3, 0.6, 0.3), specular=(0.5, 0.5, 0.5), exponent=40.0)
        elif kind == G.GLOSSY:
            mat = G.Material(G.GLOSSY, color=(0.2, 0.2, 0.6), specular=(0.6, 0.6, 0.6), exponent=30.0)
        elif kind == G.MIRROR:
            mat = G.Material(G.MIRROR, color=(0.9, 0.9, 0.9), eta=0.2, kappa=3.0)
        else:
            mat = G.Material(G.GLASS, color=(0.95, 0.95, 0.95), specular=(1.0, 1.0, 1.0), eta=1.5)
        materials.append(mat)
        meshes.append(G.Mesh(v, np.concatenate([f, np.full((len(f), 1), k, np.int32)], 1)))
        m = np.eye(4, dtype=np.float32)
        m[:3, :3] = G.rotation(rng) * rng.uniform(0.8, 1.4)
        m[:3, 3] = [(k - 2) * 2.6, 0.0, rng.uniform(-1, 1)]
        instances.append(G.Instance(k, m))
    # ground + two triangle lights in one mesh
    parts = []
    materials.append(G.Material(G.LAMBERT, color=(0.5, 0.5, 0.5)))
    parts.append((*G.quad([-20, -1.6, -20], [-20, -1.6, 20], [20, -1.6, 20], [20, -1.6, -20]), len(materials) - 1))
    lights = []
    for tri, e in (([[-3, 6, -2], [3, 6, 2], [3, 6, -2]], (30.0, 28.0, 24.0)),
                   ([[-3, 6, -2], [-3, 6, 2], [3, 6, 2]], (24.0, 28.0, 30.0))):
        materials.append(G.Material(G.EMISSIVE, color=(0, 0, 0), emission=e))
        parts.append((np.array(tri, np.float32), np.array([[0, 1, 2]], np.int32), len(materials) - 1))
        lights.append((np.array(tri[0], np.float32), np.array(tri[1], np.float32), np.array(tri[2], np.float32),
                       np.array(e, np.float32)))
    meshes.append(G._merge(parts))
    instances.append(G.Instance(len(meshes) - 1))
    cam = G.Camera(pos=(0.0, 1.5, -9.0), dir=(0.0, -0.1, 1.0), up=(0.0, 1.0, 0.0), fov=60.0, width=96, height=64)
    return G.SceneDesc(meshes, instances, materials, lights, cam, (0.4, 0.45, 0.5), "mixed")


@needs_ref
def test_reference_path_tracer_is_deterministic():
    d = small_mixed_scene()
    rs = R.RefScene(d)
    a = rs.render_pt(48, 32, 2, 5, 1234)
    b = rs.render_pt(48, 32, 2, 5, 1234)
    assert np.array_equal(a, b) and a.sum() > 0


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("w,h,spp,seed", [(64, 48, 2, 987654321), (33, 17, 3, 5)])
def test_camera_rays_bit_exact(cuda, w, h, spp, seed):
    import torch
    from imbatracer_b200.integrators import camera_matrix
    cam = G.Camera(pos=(1.0, 2.0, -7.0), dir=(-0.1, -0.2, 1.0), up=(0.0, 1.0, 0.0), fov=55.0, width=w, height=h)
    ref_rays, ref_pid, ref_sid, ref_st = R.camera_rays(w, h, spp, cam.pos, cam.dir, cam.up, cam.fov, seed)
    n = w * h * spp
    r2w = camera_matrix(cam)
    pos = np.array(cam.pos, np.float32)
    rays = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    pid = torch.zeros(n, dtype=torch.int32, device="cuda")
    sid = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(n, dtype=torch.int64, device="cuda")
    N.check(N.load().imbart_camera_rays(N.ptr(r2w), N.ptr(pos), w, h, spp, seed, 0, n, N.ptr(rays), N.ptr(pid),
                                        N.ptr(sid), N.ptr(st), None), "camera_rays")
    torch.cuda.synchronize()
    assert np.array_equal(pid.cpu().numpy(), ref_pid) and np.array_equal(sid.cpu().numpy(), ref_sid)
    assert np.array_equal(st.cpu().numpy().view(np.uint64), ref_st)
    got = rays.cpu().numpy()
    assert np.array_equal(got.view(np.int32), ref_rays.view(np.int32))


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name,w,h,spp,max_len", [
    ("config1", 64, 64, 4, 5),      # Lambertian spheres, 2-triangle area light, 4 bounces
    ("mixed", 96, 64, 8, 6),        # every material kind + constant environment
])
def test_path_tracer_image_matches_reference(cuda, name, w, h, spp, max_len):
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = small_mixed_scene() if name == "mixed" else H.scene_desc(name)
    seed = 20240611
    ref = R.RefScene(d).render_pt(w, h, spp, max_len, seed)
    gs = GpuScene(d)
    pt = PathTracer(gs, max_path_len=max_len)
    img = pt.render(spp, seed, w, h).cpu().numpy()
    err = rel_rmse(img, ref)
    assert err <= RMSE_TOL, f"relative RMSE {err:.2e}"
    assert pt.last_stats[0] >= w * h * spp and pt.last_stats[1] > 0


@needs_ref
def test_deferred_roulette_oracle_is_the_reference_at_bounce_0():
    """The oracle for rr_start (the reference's pt.cpp with its roulette call deferred,
    oracle/ref/ref_pt_rr.cpp) is the reference itself at rr_start 0, and changes the image
    when the roulette starts later."""
    rs = R.RefScene(small_mixed_scene())
    a = rs.render_pt(48, 32, 2, 5, 1234)
    assert np.array_equal(rs.render_pt_rr(48, 32, 2, 5, 0, 1234).view(np.int32), a.view(np.int32))
    assert not np.array_equal(rs.render_pt_rr(48, 32, 2, 5, 3, 1234), a)


@pytest.fixture(scope="module")
def bench_scene():
    """The benchmarked scene (200 instances of 8 meshes; Lambertian, Phong, Cook-Torrance,
    glass and mirror materials; 16 triangle lights and a constant environment) in both
    renderers."""
    from imbatracer_b200.integrators import GpuScene
    d = G.config2()
    return d, R.RefScene(d), GpuScene(d)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("rr_start", [0, 3])
def test_benchmark_frame_matches_reference(cuda, bench_scene, rr_start):
    """The benchmarked frame's settings (max_path_len 9, i.e. 8 bounces) on a 240x135 image
    of the benchmarked scene at 4 spp against the reference's PathTracer on the same seeds:
    rr_start 0 is the reference's own Russian roulette (pt.cpp:53-57), rr_start 3 the bench's
    (the reference's pt.cpp with its roulette deferred to bounce 3)."""
    from imbatracer_b200.integrators import PathTracer
    d, rs, gs = bench_scene
    w, h, spp, max_len, seed = 240, 135, 4, 9, 424242
    ref = rs.render_pt(w, h, spp, max_len, seed) if rr_start == 0 else \
        rs.render_pt_rr(w, h, spp, max_len, rr_start, seed)
    pt = PathTracer(gs, max_path_len=max_len, rr_start=rr_start)
    img = pt.render(spp, seed, w, h).cpu().numpy()
    pt.close()
    err = rel_rmse(img, ref)
    assert ref.sum() > 0 and err <= RMSE_TOL, f"relative RMSE {err:.2e}"


@pytest.mark.gpu
@needs_ref
def test_config1_full_frame_matches_reference(cuda):
    """Config 1 as specified (512x512, 1 spp, 4 bounces = max_path_len 5) against the
    reference's PathTracer on the same seeds: the frame the CPU baseline renders."""
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = G.config1(width=512, height=512)
    ref = R.RefScene(d).render_pt(512, 512, 1, 5, 31337)
    img = PathTracer(GpuScene(d), max_path_len=5).render(1, 31337, 512, 512).cpu().numpy()
    assert ref.sum() > 0
    assert rel_rmse(img, ref) <= RMSE_TOL, rel_rmse(img, ref)


@pytest.mark.gpu
@needs_ref
def test_deferred_roulette_matches_reference(cuda):
    """rr_start 2 on the scene with every material kind against the deferred-roulette oracle."""
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = small_mixed_scene()
    w, h, spp, max_len, seed = 96, 64, 8, 7, 99
    ref = R.RefScene(d).render_pt_rr(w, h, spp, max_len, 2, seed)
    img = PathTracer(GpuScene(d), max_path_len=max_len, rr_start=2).render(spp, seed, w, h).cpu().numpy()
    err = rel_rmse(img, ref)
    assert err <= RMSE_TOL, f"relative RMSE {err:.2e}"


@pytest.mark.gpu
@pytest.mark.parametrize("name,max_paths,mode", [("mixed", 0, 1), ("mixed", 0, 2), ("mixed", 10000, 2),
                                                 ("config1", 7000, 1), ("config1", 7000, 2)])
def test_graph_frames_equal_the_host_driven_loop(cuda, name, max_paths, mode):
    """The bounce loop as a CUDA graph (queue sizes read on the device, one replay per sample
    range; mode 2 with the shadow-ray work on a branch of its own) traces the same rays as the
    host-driven loop: equal ray and wavefront counts, the image equal up to the order of the
    float additions. Replays with a new seed (camera and seed are read on the device),
    rebuilds into the same executable graph (a new Russian-roulette start) and into a new one
    (a new path length) all stay equal."""
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = small_mixed_scene() if name == "mixed" else H.scene_desc("config1")
    gs = GpuScene(d)
    w, h, spp, max_len = 96, 64, 8, 6
    host = PathTracer(gs, max_path_len=max_len, rr_start=2, max_paths_in_flight=max_paths, graphs=0)
    graph = PathTracer(gs, max_path_len=max_len, rr_start=2, max_paths_in_flight=max_paths, graphs=mode)
    for seed in (11, 12, 11):
        a = host.render(spp, seed, w, h).cpu().numpy()
        b = graph.render(spp, seed, w, h).cpu().numpy()
        assert np.array_equal(host.last_stats, graph.last_stats), (host.last_stats, graph.last_stats)
        assert a.sum() > 0 and rel_rmse(b, a) <= 1e-6
    for rr, max_len in ((1, 6), (1, 4)):
        host.rr_start = graph.rr_start = rr
        host.max_path_len = graph.max_path_len = max_len
        a = host.render(spp, 13, w, h).cpu().numpy()
        b = graph.render(spp, 13, w, h).cpu().numpy()
        assert np.array_equal(host.last_stats, graph.last_stats), (host.last_stats, graph.last_stats)
        assert a.sum() > 0 and rel_rmse(b, a) <= 1e-6
    # An image accumulated over two replays equals two host frames.
    acc_h = host.render(spp, 5, w, h)
    host.render(spp, 6, w, h, image=acc_h)
    acc_g = graph.render(spp, 5, w, h)
    graph.render(spp, 6, w, h, image=acc_g)
    assert rel_rmse(acc_g.cpu().numpy(), acc_h.cpu().numpy()) <= 1e-6
    host.close()
    graph.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,kinds", [(0, 8), (1, 8), (2047, 3), (8191, 3), (8192, 8), (8193, 2), (100003, 8),
                                     (5_000_000, 7)])
def test_group_by_key_is_a_stable_counting_sort(cuda, n, kinds):
    """sort_by_material's order (ray_queue.h:211-244) as the permutation the wavefront
    kernels shade through: equal to a stable sort of the keys, on ragged tile counts, a
    single entry, empty queues and keys absent from the queue."""
    import torch
    rng = np.random.default_rng(n + kinds)
    keys = rng.integers(0, kinds, n).astype(np.uint8)
    if n > 10:
        keys[rng.random(n) < 0.6] = kinds - 1          # one dominant key, as in real wavefronts
    k = torch.from_numpy(keys).cuda()
    perm = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    N.check(N.load().imbart_group_by_key(N.ptr(k) if n else None, n, N.ptr(perm), None), "imbart_group_by_key")
    torch.cuda.synchronize()
    got = perm.cpu().numpy()[:n]
    assert np.array_equal(got, np.argsort(keys, kind="stable").astype(np.int32))
    if n > 10:
        # Keys above 7 are grouped with 7: still a permutation, nothing written out of range.
        wild = keys.copy()
        wild[::7] = 200
        k2 = torch.from_numpy(wild).cuda()
        N.check(N.load().imbart_group_by_key(N.ptr(k2), n, N.ptr(perm), None), "imbart_group_by_key")
        torch.cuda.synchronize()
        assert np.array_equal(perm.cpu().numpy()[:n], np.argsort(np.minimum(wild, 7), kind="stable").astype(np.int32))


@pytest.mark.gpu
def test_graph_frames_edge_cases(cuda):
    """Graph-driven frames at the edges: one pixel and one sample, camera rays only
    (max_path_len 1: no continuation, shadow rays only), wavefronts of one path, and a
    frame whose last sample range holds a single path; each equals the host-driven loop."""
    from imbatracer_b200.integrators import GpuScene, PathTracer
    gs = GpuScene(small_mixed_scene())
    cases = [(1, 1, 1, 6, 0), (16, 8, 2, 1, 0), (5, 3, 2, 4, 1), (9, 7, 3, 5, 47), (9, 7, 3, 5, 94)]
    for w, h, spp, max_len, max_paths in cases:
        host = PathTracer(gs, max_path_len=max_len, max_paths_in_flight=max_paths, graphs=0)
        graph = PathTracer(gs, max_path_len=max_len, max_paths_in_flight=max_paths, graphs=2)
        a = host.render(spp, 3, w, h).cpu().numpy()
        b = graph.render(spp, 3, w, h).cpu().numpy()
        assert np.array_equal(host.last_stats, graph.last_stats), (w, h, spp, max_len, max_paths)
        den = max(float(np.sqrt(np.mean(a.astype(np.float64) ** 2))), 1e-30)
        assert float(np.sqrt(np.mean((b.astype(np.float64) - a) ** 2))) / den <= 1e-6
        host.close()
        graph.close()
    # Without statistics the call does not synchronize; the stream orders the image read.
    pt = PathTracer(gs, max_path_len=5, graphs=2)
    a = pt.render(4, 8, 40, 30).cpu().numpy()
    b = pt.render(4, 8, 40, 30, stats=False).cpu().numpy()
    assert a.sum() > 0 and rel_rmse(b, a) <= 1e-6


@pytest.mark.gpu
def test_graph_frames_beside_device_wide_synchronization(cuda):
    """A thread that renders graph-driven frames while another thread creates scenes (whose
    set-up synchronizes the whole device): both succeed, and the frames equal the same frames
    rendered alone. (Graphs are built with the graph API, not by stream capture, which such a
    synchronization would invalidate.)"""
    import threading
    import torch
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = small_mixed_scene()
    gs = GpuScene(d)
    alone = [PathTracer(gs, max_path_len=5, graphs=2).render(2, 100 + k, 48, 32).cpu().numpy() for k in range(6)]
    out, errors = [], []

    def render():
        try:
            torch.cuda.set_device(0)
            pt = PathTracer(gs, max_path_len=5, graphs=2)
            for k in range(6):
                pt.render(2, 100 + k, 48, 32, cam=None)   # a fresh image (new graph) every frame
                out.append(pt.render(2, 100 + k, 48, 32).cpu().numpy())
        except Exception as e:  # reported below
            errors.append(e)

    t = threading.Thread(target=render)
    t.start()
    scenes = []
    while t.is_alive():
        scenes.append(GpuScene(d))
        torch.cuda.synchronize()
    t.join()
    assert not errors, errors
    assert len(scenes) >= 1 and len(out) == 6
    for a, b in zip(alone, out):
        assert rel_rmse(b, a) <= 1e-6
