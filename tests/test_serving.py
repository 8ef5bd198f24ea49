"""The request server (imbart_server_*): merged wavefronts over several resident scenes,
VCM-family frames between them.

A render served in a mix of other requests must give the image the single-request path
(imbart_pt_render) gives alone: paths are seeded per sample and shaded by the same code, so
only the order of the float additions into the image differs (tolerance: relative RMSE
1e-5). Ray batches must return exactly the hits of imbart_trace. Eviction under a small
pool must not change results.
"""
import numpy as np
import pytest

from imbatracer_b200 import native as N
from imbatracer_b200 import scenegen as G
from tests import helpers as H
from tests.test_pt import small_mixed_scene

MIX_TOL = 1e-5


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / max(np.sqrt(np.mean(b.astype(np.float64) ** 2)),
                                                                          1e-30))


def sphere_scene(seed, n, level):
    return G._sphere_field(seed, n, level, 64, 64, f"spheres{seed}")


@pytest.fixture(scope="module")
def scenes():
    from imbatracer_b200 import scene as S
    out = []
    for d in (small_mixed_scene(), sphere_scene(3, 6, 2), sphere_scene(4, 10, 3)):
        out.append((d, S.build_traversal_data(d.meshes, d.instances)))
    return out


def plain_image(d, td, w, h, spp, max_len, seed, rr_start=0):
    from imbatracer_b200.integrators import GpuScene, PathTracer
    gs = GpuScene(d, td=td)
    pt = PathTracer(gs, max_path_len=max_len, rr_start=rr_start)
    img = pt.render(spp, seed, w, h).cpu().numpy()
    pt.close()
    gs.close()
    return img


REQS = [  # (scene index, width, height, spp, max_path_len, seed, rr_start)
    (0, 48, 32, 4, 6, 11, 0),
    (1, 40, 40, 2, 5, 12, 2),
    (2, 64, 48, 3, 5, 13, 0),
    (0, 17, 9, 5, 4, 14, 1),
    (1, 1, 1, 7, 3, 15, 0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_renders_in_a_mix_match_single_request_path(cuda, scenes, mode):
    from imbatracer_b200.serving import Server
    srv = Server(mode=mode, hbm_budget=256 << 20, max_paths=20000)
    ids = [srv.add_scene(d, td) for d, td in scenes]
    tickets = []
    for si, w, h, spp, ml, seed, rr in REQS:
        d = scenes[si][0]
        tickets.append(srv.submit_render(ids[si], d.camera, w, h, spp, ml, seed, rr_start=rr))
    for (t, img), (si, w, h, spp, ml, seed, rr) in zip(tickets, REQS):
        res = srv.wait(t)
        assert res["status"] == 0 and res["done_ms"] >= res["start_ms"] >= res["submit_ms"]
        d, td = scenes[si]
        ref = plain_image(d, td, w, h, spp, ml, seed, rr)
        assert rel_rmse(img, ref) <= MIX_TOL, (si, w, h, rel_rmse(img, ref))
    st = srv.stats()
    assert st["completed"] == len(REQS) and st["failed"] == 0
    if mode == "batched":
        # Several requests shared wavefronts: far fewer waves than the requests' own sum.
        assert st["waves"] < sum(r[4] for r in REQS) * 2
    srv.close()


@pytest.mark.gpu
def test_render_alone_equals_render_in_mix(cuda, scenes):
    from imbatracer_b200.serving import Server
    d, td = scenes[2]
    alone = Server(hbm_budget=256 << 20, max_paths=8192)
    sid = alone.add_scene(d, td)
    t, img_alone = alone.submit_render(sid, d.camera, 64, 48, 4, 5, 99)
    assert alone.wait(t)["status"] == 0
    alone.close()
    mix = Server(hbm_budget=256 << 20, max_paths=8192)
    ids = [mix.add_scene(dd, tt) for dd, tt in scenes]
    others = [mix.submit_render(ids[k % 3], scenes[k % 3][0].camera, 32, 32, 2, 5, 500 + k) for k in range(6)]
    t, img_mix = mix.submit_render(ids[2], d.camera, 64, 48, 4, 5, 99)
    rays = G.random_rays(np.random.default_rng(1), 5000, -12, 12)
    hits = np.zeros(len(rays), N.HIT_DTYPE)
    tr = mix.submit_rays(ids[0], rays, hits)
    assert mix.wait(t)["status"] == 0
    for tt, _ in others:
        assert mix.wait(tt)["status"] == 0
    assert mix.wait(tr)["status"] == 0
    mix.close()
    assert rel_rmse(img_mix, img_alone) <= MIX_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("where", ["pageable", "pinned", "device"])
def test_ray_batches_bit_exact(cuda, scenes, where):
    import torch
    from imbatracer_b200 import scene as S
    from imbatracer_b200.serving import Server
    srv = Server(hbm_budget=256 << 20, max_paths=30000)   # batches larger than a wavefront are split
    ids = [srv.add_scene(d, td) for d, td in scenes]
    rng = np.random.default_rng(7)
    jobs = []
    for k, (d, td) in enumerate(scenes):
        for flags in (N.TRACE_CLOSEST, N.TRACE_ANY):
            n = int(rng.integers(1, 70000))
            rays = G.random_rays(rng, n, -12, 12)
            if flags == N.TRACE_ANY:
                rays["dir"][:, 3] = rng.uniform(0.1, 30.0, n).astype(np.float32)
            ds = S.DeviceScene(td)
            want = np.zeros(n, N.HIT_DTYPE)
            ds.trace_host(rays, want, any_hit=flags == N.TRACE_ANY)
            ds.close()
            if where == "pageable":
                r_in, h_out = rays, np.zeros(n, N.HIT_DTYPE)
            elif where == "pinned":
                r_in = torch.from_numpy(rays.view(np.float32).reshape(n, 8)).pin_memory()
                h_out = torch.zeros((n, 4), dtype=torch.int32).pin_memory()
            else:
                r_in = torch.from_numpy(rays.view(np.float32).reshape(n, 8)).cuda()
                h_out = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
            jobs.append((srv.submit_rays(ids[k], r_in, h_out, flags), h_out, want, flags))
    for t, h_out, want, flags in jobs:
        assert srv.wait(t)["status"] == 0
        got = h_out if isinstance(h_out, np.ndarray) else h_out.cpu().numpy().view(N.HIT_DTYPE).reshape(-1)
        if flags == N.TRACE_CLOSEST:
            assert H.hits_equal(got, want).all()
        else:
            assert np.array_equal(got["tri_id"] >= 0, want["tri_id"] >= 0)
    srv.close()


VCM_REQS = [  # (scene index, algorithm, width, height, iterations, max_path_len, light seed, camera seed)
    (0, "vcm", 40, 32, 2, 5, 101, 201),
    (1, "bpt", 32, 24, 2, 5, 102, 202),
    (2, "ppm", 24, 24, 3, 5, 103, 203),
    (0, "lt", 48, 32, 2, 4, 104, 204),
    (1, "pt", 16, 12, 2, 4, 105, 205),
]
SEED_STEP = 7
TILE_STEP = 0x9E3779B9


def vcm_alone(d, td, algo, w, h, iters, ml, ls, cs):
    """The same frame through VcmIntegrator alone: iteration i seeded ls / cs + (i - 1) * 7."""
    from imbatracer_b200.integrators import GpuScene, VcmIntegrator
    gs = GpuScene(d, td=td)
    vi = VcmIntegrator(gs, algo, w, h, max_path_len=ml)
    img = None
    for i in range(iters):
        img = vi.render(i + 1, ls + i * SEED_STEP, cs + i * SEED_STEP, TILE_STEP, image=img)
    out = img.cpu().numpy()
    vi.close()
    gs.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_vcm_family_requests_in_a_mix(cuda, scenes, mode):
    """VCM, BPT, PPM, LT and VCM-PT frames served between merged path-tracing wavefronts
    give the images of VcmIntegrator alone, and the renders beside them are unchanged."""
    from imbatracer_b200.serving import Server
    srv = Server(mode=mode, hbm_budget=256 << 20, max_paths=20000)
    ids = [srv.add_scene(d, td) for d, td in scenes]
    vt, rt = [], []
    for k, (si, algo, w, h, it, ml, ls, cs) in enumerate(VCM_REQS):
        d = scenes[si][0]
        vt.append(srv.submit_vcm(ids[si], d.camera, w, h, algo, iterations=it, max_path_len=ml, light_seed=ls,
                                 camera_seed=cs, seed_step=SEED_STEP, light_seed_step=TILE_STEP))
        si2, w2, h2, spp, ml2, seed, rr = REQS[k]
        rt.append(srv.submit_render(ids[si2], scenes[si2][0].camera, w2, h2, spp, ml2, seed, rr_start=rr))
    for (t, img), (si, algo, w, h, it, ml, ls, cs) in zip(vt, VCM_REQS):
        res = srv.wait(t)
        assert res["status"] == 0 and res["kind"] == 2
        d, td = scenes[si]
        ref = vcm_alone(d, td, algo, w, h, it, ml, ls, cs)
        assert ref.sum() > 0
        assert rel_rmse(img, ref) <= MIX_TOL, (algo, rel_rmse(img, ref))
    for (t, img), (si, w, h, spp, ml, seed, rr) in zip(rt, REQS):
        assert srv.wait(t)["status"] == 0
        d, td = scenes[si]
        assert rel_rmse(img, plain_image(d, td, w, h, spp, ml, seed, rr)) <= MIX_TOL
    st = srv.stats()
    assert st["completed"] == len(VCM_REQS) + len(REQS) and st["failed"] == 0
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["vcm", "bpt"])
def test_one_long_vcm_request_spread_over_lanes(cuda, scenes, algo):
    """A VCM-family request with many iterations and nothing beside it: the server's lanes
    render its iterations concurrently (iterations depend on their index only), and the image
    equals VcmIntegrator's iterations run one after another (up to the order of the float
    additions); its photon radius is estimated once, before the other lanes join."""
    from imbatracer_b200.serving import Server
    srv = Server(mode="batched", hbm_budget=256 << 20, max_paths=20000)
    ids = [srv.add_scene(d, td) for d, td in scenes]
    d, td = scenes[1]
    t, img = srv.submit_vcm(ids[1], d.camera, 40, 30, algo, iterations=12, max_path_len=5, light_seed=11,
                            camera_seed=22, seed_step=SEED_STEP, light_seed_step=TILE_STEP)
    res = srv.wait(t)
    assert res["status"] == 0 and res["kind"] == 2
    ref = vcm_alone(d, td, algo, 40, 30, 12, 5, 11, 22)
    assert ref.sum() > 0 and rel_rmse(img, ref) <= MIX_TOL, rel_rmse(img, ref)
    assert srv.stats()["failed"] == 0
    srv.close()


@pytest.mark.gpu
def test_vcm_request_validation(cuda, scenes):
    from imbatracer_b200.serving import Server
    srv = Server(hbm_budget=64 << 20, max_paths=4096)
    sid = srv.add_scene(*scenes[0])
    d = scenes[0][0]
    with pytest.raises(N.ImbartError):
        srv.submit_vcm(sid, d.camera, 8, 8, "vcm", iterations=0)
    with pytest.raises(N.ImbartError):
        srv.submit_vcm(sid, d.camera, 8, 8, "vcm", num_knn=65)
    with pytest.raises(N.ImbartError):
        srv.submit_vcm(sid, d.camera, 8, 8, "vcm", radius_factor=0.0)
    t, img = srv.submit_vcm(sid, d.camera, 8, 8, "bpt", base_radius=0.05)
    assert srv.wait(t)["status"] == 0 and img.sum() > 0
    srv.close()


@pytest.mark.gpu
def test_lru_eviction_keeps_results(cuda, scenes):
    from imbatracer_b200.serving import Server
    probe = Server(hbm_budget=256 << 20, max_paths=4096)
    ids = [probe.add_scene(d, td) for d, td in scenes]
    sizes = []
    for k in range(3):
        before = probe.stats()["pool_used_bytes"]
        t, _ = probe.submit_render(ids[k], scenes[k][0].camera, 1, 1, 1, 2, 1)
        probe.wait(t)
        sizes.append(probe.stats()["pool_used_bytes"] - before)
    probe.close()
    # Room for the largest scene plus an image, not for two scenes at once.
    assert min(sizes) >= 32 << 10
    budget = max(sizes) + min(sizes) // 2
    srv = Server(hbm_budget=budget, max_paths=4096)
    ids = [srv.add_scene(d, td) for d, td in scenes]
    order = [0, 1, 2, 0, 2, 1]
    imgs = []
    for k in order:          # one at a time, so every switch of scene evicts
        t, img = srv.submit_render(ids[k], scenes[k][0].camera, 24, 16, 2, 4, 70 + k)
        assert srv.wait(t)["status"] == 0
        imgs.append(img)
    st = srv.stats()
    assert st["scene_evictions"] >= len(order) - 1 and st["scene_uploads"] >= len(order)
    for k, img in zip(order, imgs):
        d, td = scenes[k]
        assert rel_rmse(img, plain_image(d, td, 24, 16, 2, 4, 70 + k)) <= MIX_TOL
    srv.close()


@pytest.mark.gpu
def test_scene_larger_than_pool_is_refused(cuda, scenes):
    from imbatracer_b200.serving import Server
    srv = Server(hbm_budget=64 << 10, max_paths=1024)
    d, td = scenes[2]
    with pytest.raises(N.ImbartError):
        srv.add_scene(d, td)
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_scenes_registered_through_the_gpu_builder(cuda, scenes, mode):
    """imbart_server_add_scene_gpu_build (traversal arrays built on the GPU, kept on the host
    like a converted scene's): renders equal the single-request path's on the host-built
    scene (hits do not depend on the tree) and ray batches equal imbart_trace's hits."""
    from imbatracer_b200 import scene as S
    from imbatracer_b200.serving import Server
    srv = Server(mode=mode, hbm_budget=64 << 20, max_paths=1 << 16)
    ids = []
    for d, _ in scenes:
        ids.append(srv.add_scene(d, gpu_build=True))
        assert srv.last_build_ms > 0
    tickets = []
    for k, (si, w, h, spp, ml, seed, rr) in enumerate(REQS):
        d, td = scenes[si]
        t, img = srv.submit_render(ids[si], d.camera, w, h, spp, ml, seed, rr_start=rr)
        tickets.append((t, img, plain_image(d, td, w, h, spp, ml, seed, rr), k))
    d, td = scenes[2]
    lo, hi = G.scene_box(d)
    rays = G.random_rays(np.random.default_rng(3), 5000, lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo))
    hits = np.zeros(len(rays), N.HIT_DTYPE)
    tb = srv.submit_rays(ids[2], rays, hits)
    for t, img, want, k in tickets:
        assert srv.wait(t)["status"] == 0
        assert rel_rmse(img, want) <= MIX_TOL, (k, rel_rmse(img, want))
    assert srv.wait(tb)["status"] == 0
    ds = S.DeviceScene(td)
    ref = np.zeros_like(hits)
    ds.trace_host(rays, ref)
    assert (ref["tri_id"] >= 0).sum() > 500
    assert np.array_equal(hits.view(np.int32), ref.view(np.int32))
    srv.close()
