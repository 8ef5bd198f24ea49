"""GPU parity of the traversal kernels against the oracle, through the C ABI.

Closest hits must match the oracle bit for bit (triangle id, instance id, t, u, and v through
imbart_trace_uv): the kernel evaluates the same watertight test with the same rounding, and
equal-t hits resolve to the smallest (inst_id, tri_id). Any-hit queries must agree on
occlusion. The statistics variant must report exactly the work the restated walk counts.
"""
import numpy as np
import pytest

from imbatracer_b200 import native as N
from imbatracer_b200 import scene as S
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def to_dev(arr, torch, dev):
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8)).to(dev)


def run_gpu(ds, rays, any_hit=False, stats=False):
    import torch
    dev = torch.device("cuda:0")
    d_rays = to_dev(rays, torch, dev)
    d_hits = torch.zeros(len(rays) * 16, dtype=torch.uint8, device=dev)
    d_v = torch.zeros(len(rays), dtype=torch.float32, device=dev)
    lib = N.load()
    flags = N.TRACE_ANY if any_hit else N.TRACE_CLOSEST
    st = None
    if stats:
        st = torch.zeros(3, dtype=torch.int64, device=dev)
        N.check(lib.imbart_trace_stats(ds.handle, N.ptr(d_rays), N.ptr(d_hits), len(rays), flags, N.ptr(st), None),
                "trace_stats")
    else:
        N.check(lib.imbart_trace_uv(ds.handle, N.ptr(d_rays), N.ptr(d_hits), N.ptr(d_v), len(rays), flags, None),
                "trace")
    torch.cuda.synchronize()
    hits = d_hits.cpu().numpy().view(N.HIT_DTYPE)
    return hits, d_v.cpu().numpy(), (st.cpu().numpy() if st is not None else None)


@pytest.mark.parametrize("name,n", [("tiny", 4000), ("config1", 200000), ("config2", 200000)])
def test_closest_hit_bit_exact(cuda, name, n):
    td = H.traversal_data(name)
    ds = S.DeviceScene(td)
    rays = H.ray_set(name, n, seed=3)
    ref, ref_v = O.trace_node2(td, rays, with_v=True)
    hits, v, _ = run_gpu(ds, rays)
    eq = H.hits_equal(ref, hits)
    bad = np.nonzero(~eq)[0]
    assert eq.all(), f"{len(bad)} of {len(rays)} differ, e.g. {ref[bad[:3]]} vs {hits[bad[:3]]}"
    assert np.array_equal(ref_v.view(np.int32), v.view(np.int32))
    assert (ref["tri_id"] >= 0).mean() > 0.1
    assert N.load().imbart_scene_error_count(ds.handle) == 0


@pytest.mark.parametrize("name", ["tiny", "config1", "config2"])
def test_any_hit_occlusion(cuda, name):
    td = H.traversal_data(name)
    ds = S.DeviceScene(td)
    rays = H.ray_set(name, 100000, seed=4)
    # shadow-style rays: bounded segments
    rays["dir"][: len(rays) // 2, 3] = np.float32(5.0)
    ref = O.trace_node2(td, rays, any_hit=True)
    hits, _, _ = run_gpu(ds, rays, any_hit=True)
    assert np.array_equal(ref["tri_id"] >= 0, hits["tri_id"] >= 0)
    occ = hits["tri_id"] >= 0
    # a reported occluder lies within the segment
    t = hits["tmax"][occ]
    assert (t >= rays["org"][occ, 3]).all() and (t <= rays["dir"][occ, 3]).all()


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_stats_match_restated_walk(cuda, name):
    """The kernel's node/triangle/instance counts equal the restated walk's, ray for ray in
    aggregate: the bytes used for the roofline are the bytes the kernel fetches."""
    td = H.traversal_data(name)
    ds = S.DeviceScene(td)
    wn, wt, wi, root = H.wide_arrays(td)
    rays = H.ray_set(name, 50000, seed=5)
    for any_hit in (False, True):
        hits, _, st = run_gpu(ds, rays, any_hit=any_hit, stats=True)
        hw, nbytes, counts = O.wide_walk(wn, wt, wi, root, rays, any_hit=any_hit)
        assert np.array_equal(st, counts), (st, counts)
        if not any_hit:
            assert H.hits_equal(hw, hits).all()


def test_dropin_device_entry_points(cuda):
    """intersect_/occluded_gpu_masked_instanced with device buffers in the reference layout."""
    import torch
    td = H.traversal_data("config1")
    dev = torch.device("cuda:0")
    lib = N.load()
    lib.imbart_invalidate_scenes()
    d_nodes = to_dev(td.nodes, torch, dev)
    d_insts = to_dev(td.instances, torch, dev)
    d_tris = to_dev(td.tris, torch, dev)
    d_idx = to_dev(td.indices, torch, dev)
    d_tc = to_dev(td.texcoords, torch, dev)
    d_masks = to_dev(td.masks, torch, dev)
    d_mb = to_dev(td.mask_buffer, torch, dev)
    rays = H.ray_set("config1", 65536, seed=6)
    count = (len(rays) + 63) // 64 * 64
    padded = np.zeros(count, N.RAY_DTYPE)
    padded[: len(rays)] = rays
    d_rays = to_dev(padded, torch, dev)
    d_hits = torch.zeros(count * 16, dtype=torch.uint8, device=dev)
    args = (td.root, N.ptr(d_nodes), N.ptr(d_insts), N.ptr(d_tris), N.ptr(d_rays), N.ptr(d_hits), N.ptr(d_idx),
            N.ptr(d_tc), N.ptr(d_masks), N.ptr(d_mb), count)
    lib.imbart_clear_error()
    lib.intersect_gpu_masked_instanced(*args)
    assert N.last_error()[0] == 0, N.last_error()
    hits = d_hits.cpu().numpy().view(N.HIT_DTYPE)
    ref = O.trace_node2(td, padded)
    assert H.hits_equal(ref, hits).all()
    assert (hits["tri_id"][len(rays):] == -1).all()     # zeroed padding rays miss
    lib.occluded_gpu_masked_instanced(*args)
    assert N.last_error()[0] == 0
    occ = d_hits.cpu().numpy().view(N.HIT_DTYPE)
    refa = O.trace_node2(td, padded, any_hit=True)
    assert np.array_equal(refa["tri_id"] >= 0, occ["tri_id"] >= 0)
    lib.imbart_invalidate_scenes()


@pytest.mark.skipif(not __import__("oracle.refwrap", fromlist=["x"]).available(), reason="oracle/_ref not built")
def test_dropin_with_reference_sbvh_layout(cuda):
    """The reference's own SBVH/binned adapters' output, uploaded to device buffers the way
    Scene::upload_* does, traced through intersect_gpu_masked_instanced."""
    import torch
    from tests.test_reference_pins import ref_traversal_data
    td = ref_traversal_data(H.scene_desc("config1"))
    lib = N.load()
    lib.imbart_invalidate_scenes()
    dev = torch.device("cuda:0")
    bufs = [to_dev(a, torch, dev) for a in (td.nodes, td.instances, td.tris, td.indices, td.texcoords, td.masks,
                                            td.mask_buffer)]
    rays = H.ray_set("config1", 30000, seed=12)
    count = (len(rays) + 63) // 64 * 64
    padded = np.zeros(count, N.RAY_DTYPE)
    padded[: len(rays)] = rays
    d_rays = to_dev(padded, torch, dev)
    d_hits = torch.zeros(count * 16, dtype=torch.uint8, device=dev)
    lib.imbart_clear_error()
    lib.intersect_gpu_masked_instanced(td.root, N.ptr(bufs[0]), N.ptr(bufs[1]), N.ptr(bufs[2]), N.ptr(d_rays),
                                       N.ptr(d_hits), N.ptr(bufs[3]), N.ptr(bufs[4]), N.ptr(bufs[5]), N.ptr(bufs[6]),
                                       count)
    assert N.last_error()[0] == 0, N.last_error()
    hits = d_hits.cpu().numpy().view(N.HIT_DTYPE)
    assert H.hits_equal(O.trace_node2(td, padded), hits).all()
    lib.imbart_invalidate_scenes()


def test_host_buffer_trace(cuda):
    td = H.traversal_data("config2")
    ds = S.DeviceScene(td)
    rays = H.ray_set("config2", 30000, seed=7)
    hits = np.zeros(len(rays), N.HIT_DTYPE)
    ds.trace_host(rays, hits)
    assert H.hits_equal(O.trace_node2(td, rays), hits).all()


def masked_config1(two_level: bool = False):
    """config1's spheres with checkerboard opacity masks on every other sphere material and a
    single transparent texel on the ground; two_level adds a second, translated instance of
    the mesh (a two-level scene instead of one identity instance)."""
    d = H.scene_desc("config1")
    mesh = d.meshes[0]
    rng = np.random.default_rng(8)
    tc = rng.uniform(-1.5, 1.5, size=(len(mesh.vertices), 2)).astype(np.float32)
    m2 = S.Mesh(mesh.vertices, mesh.indices, mesh.normals, tc, mesh.geom_normals)
    n_mats = int(mesh.indices[:, 3].max()) + 1
    masks = np.zeros(n_mats, N.MASK_DTYPE)
    masks["width"] = 1
    masks["height"] = 1
    buf = [1, 1, 1, 1]
    checker = (np.indices((8, 8)).sum(0) % 2).astype(np.uint8).reshape(-1)
    for m in range(0, n_mats - 3, 2):       # every other sphere material gets the checkerboard
        masks[m] = (8, 8, len(buf))
        buf += checker.tolist()
    masks[n_mats - 3] = (1, 1, len(buf))    # the ground: a single transparent texel
    buf.append(0)
    insts = list(d.instances)
    if two_level:
        t = np.eye(4, dtype=np.float32)
        t[:3, 3] = [3.0, 0.5, -2.0]
        insts.append(S.Instance(0, t))
    return S.build_traversal_data([m2], insts, masks=masks, mask_buffer=np.array(buf, np.uint8))


def test_alpha_masks(cuda):
    """Checkerboard opacity masks on config1's sphere materials: transparent texels let rays
    through; GPU and oracle agree bit for bit."""
    td = masked_config1()
    ds = S.DeviceScene(td)
    assert ds.info.masked == 1
    rays = H.ray_set("config1", 100000, seed=9)
    ref = O.trace_node2(td, rays)
    hits, _, _ = run_gpu(ds, rays)
    assert H.hits_equal(ref, hits).all()
    unmasked = O.trace_node2(H.traversal_data("config1"), rays)
    assert (unmasked["tri_id"] != ref["tri_id"]).sum() > 100   # the masks matter
    refa = O.trace_node2(td, rays, any_hit=True)
    occ, _, _ = run_gpu(ds, rays, any_hit=True)
    assert np.array_equal(refa["tri_id"] >= 0, occ["tri_id"] >= 0)


@pytest.mark.parametrize("two_level,width", [(False, 8), (True, 8), (False, 4), (True, 4)])
def test_alpha_masks_every_kernel_variant(cuda, two_level, width):
    """The masked kernels of every shape (flat kernels for the single identity instance,
    two-level ones with a second instance; 8- and 4-wide trees) give the oracle's closest hits
    bit for bit and its occlusion answers."""
    lib = N.load()
    saved = S.trace_config_snapshot()
    try:
        td = masked_config1(two_level)
        ds = S.DeviceScene(td, node_width=width)
        assert ds.info.masked == 1 and ds.node_width == width
        rays = H.ray_set("config1", 20000, seed=29)
        ref = O.trace_node2(td, rays)
        refa = O.trace_node2(td, rays, any_hit=True)
        for variant in range(18):
            for flags in (N.TRACE_CLOSEST, N.TRACE_ANY):
                N.check(lib.imbart_set_trace_class(flags, variant, 16), "imbart_set_trace_class")
            hits, _, _ = run_gpu(ds, rays)
            assert H.hits_equal(ref, hits).all(), variant
            occ, _, _ = run_gpu(ds, rays, any_hit=True)
            assert np.array_equal(refa["tri_id"] >= 0, occ["tri_id"] >= 0), variant
        assert lib.imbart_scene_error_count(ds.handle) == 0
        ds.close()
    finally:
        S.trace_config_restore(saved)


def test_empty_and_zero_count(cuda):
    import torch
    ds = S.DeviceScene(H.traversal_data("tiny"))
    lib = N.load()
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert lib.imbart_trace(ds.handle, N.ptr(d), N.ptr(d), 0, 0, None) == 0
    assert lib.imbart_trace(ds.handle, N.ptr(d), N.ptr(d), -1, 0, None) == 1


def test_autotuner_picks_a_configuration_and_hits_stay_exact(cuda):
    """imbart_trace_autotune times the persistent-kernel configurations of a query class and
    keeps the fastest; the hits of every class stay bit-exact afterwards."""
    import ctypes as C
    import torch
    lib = N.load()
    saved = {}
    for flags in (N.TRACE_CLOSEST, N.TRACE_ANY, N.TRACE_CLOSEST | N.TRACE_COHERENT):
        v, r = C.c_int(0), C.c_int(0)
        lib.imbart_get_trace_class(flags, C.byref(v), C.byref(r))
        saved[flags] = (v.value, r.value, lib.imbart_get_trace_tri_batch(flags))
    try:
        td = H.traversal_data("config2")
        ds = S.DeviceScene(td)
        rays = H.ray_set("config2", 50000, seed=12)
        dev = torch.device("cuda:0")
        d_rays = to_dev(rays, torch, dev)
        d_hits = torch.zeros(len(rays) * 16, dtype=torch.uint8, device=dev)
        for flags in saved:
            t = N.TraceTuning()
            N.check(lib.imbart_trace_autotune(ds.handle, N.ptr(d_rays), N.ptr(d_hits), len(rays), flags, None,
                                              C.byref(t)), "autotune")
            assert 1 <= t.variant <= 17 and t.refill in (4, 8, 16, 24, 32) and 0 < t.ms <= t.default_ms * 1.0001
            v, r = C.c_int(0), C.c_int(0)
            lib.imbart_get_trace_class(flags, C.byref(v), C.byref(r))
            assert (v.value, r.value) == (t.variant, t.refill)
            assert lib.imbart_get_trace_tri_batch(flags) == t.tri_batch and 0 <= t.tri_batch <= 4
        ref = O.trace_node2(td, rays)
        hits, _, _ = run_gpu(ds, rays)
        assert H.hits_equal(ref, hits).all()
        refa = O.trace_node2(td, rays, any_hit=True)
        hitsa, _, _ = run_gpu(ds, rays, any_hit=True)
        assert np.array_equal(refa["tri_id"] >= 0, hitsa["tri_id"] >= 0)
        assert lib.imbart_trace_autotune(ds.handle, N.ptr(d_rays), N.ptr(d_hits), 0, 0, None, None) != 0
        lib.imbart_clear_error()
    finally:
        for flags, (v, r, b) in saved.items():
            lib.imbart_set_trace_class(flags, v, r)
            lib.imbart_set_trace_tri_batch(flags, b)


@pytest.mark.gpu
def test_every_kernel_variant_is_exact(cuda):
    """Each traversal kernel shape the autotuner may pick (0: one ray per thread, 1..10:
    persistent warps at different block sizes, blocks per SM and shared stack depths, 11..17:
    the same with the cooperative triangle phase; with triangle batches 0, 1 and 2, which the
    cooperative shapes ignore) gives the
    oracle's closest hits bit for bit, its occlusion answers, and the restated walk's node,
    triangle and instance counts."""
    import ctypes as C
    lib = N.load()
    saved = {}
    for flags in (N.TRACE_CLOSEST, N.TRACE_ANY):
        v, r = C.c_int(0), C.c_int(0)
        lib.imbart_get_trace_class(flags, C.byref(v), C.byref(r))
        saved[flags] = (v.value, r.value, lib.imbart_get_trace_tri_batch(flags))
    try:
        td = H.traversal_data("config2")
        ds = S.DeviceScene(td)
        rays = H.ray_set("config2", 20000, seed=21)
        ref = O.trace_node2(td, rays)
        refa = O.trace_node2(td, rays, any_hit=True)
        wn, wt, wi, root = H.wide_arrays(td)
        counts = {a: O.wide_walk(wn, wt, wi, root, rays, any_hit=a)[2] for a in (False, True)}
        for variant in range(18):
            for tri_batch in (0, 1, 2):
                for flags in saved:
                    N.check(lib.imbart_set_trace_class(flags, variant, 16), "imbart_set_trace_class")
                    N.check(lib.imbart_set_trace_tri_batch(flags, tri_batch), "imbart_set_trace_tri_batch")
                hits, _, _ = run_gpu(ds, rays)
                assert H.hits_equal(ref, hits).all(), (variant, tri_batch)
                hitsa, _, _ = run_gpu(ds, rays, any_hit=True)
                assert np.array_equal(refa["tri_id"] >= 0, hitsa["tri_id"] >= 0), (variant, tri_batch)
                for a in (False, True):
                    _, _, st = run_gpu(ds, rays, any_hit=a, stats=True)
                    assert np.array_equal(st, counts[a]), (variant, tri_batch, a, st, counts[a])
        assert lib.imbart_set_trace_class(N.TRACE_CLOSEST, 18, 16) != 0
        assert lib.imbart_set_trace_tri_batch(N.TRACE_CLOSEST, -1) != 0
        lib.imbart_clear_error()
    finally:
        for flags, (v, r, b) in saved.items():
            lib.imbart_set_trace_class(flags, v, r)
            lib.imbart_set_trace_tri_batch(flags, b)


@pytest.mark.gpu
def test_four_wide_scene_every_variant_is_exact(cuda):
    """A scene converted 4-wide runs the 4-slot kernels (every shape, triangle batches 0 and 1)
    and gives the oracle's closest hits bit for bit, its occlusion answers, and the restated
    walk's counts over the 4-wide tree."""
    import ctypes as C
    lib = N.load()
    saved = S.trace_config_snapshot()
    try:
        td = H.traversal_data("config2")
        ds = S.DeviceScene(td, node_width=4)
        assert ds.node_width == 4 and lib.imbart_get_node_width() == 8
        rays = H.ray_set("config2", 20000, seed=23)
        ref = O.trace_node2(td, rays)
        refa = O.trace_node2(td, rays, any_hit=True)
        wn, wt, wi, root = H.wide_arrays(td, node_width=4)
        assert ds.info.wide_nodes == len(wn)
        counts = {a: O.wide_walk(wn, wt, wi, root, rays, any_hit=a)[2] for a in (False, True)}
        for variant in range(18):
            for tri_batch in (0, 1):
                for flags in (N.TRACE_CLOSEST, N.TRACE_ANY):
                    N.check(lib.imbart_set_trace_class(flags, variant, 16), "imbart_set_trace_class")
                    N.check(lib.imbart_set_trace_tri_batch(flags, tri_batch), "imbart_set_trace_tri_batch")
                hits, v, _ = run_gpu(ds, rays)
                assert H.hits_equal(ref, hits).all(), (variant, tri_batch)
                hitsa, _, _ = run_gpu(ds, rays, any_hit=True)
                assert np.array_equal(refa["tri_id"] >= 0, hitsa["tri_id"] >= 0), (variant, tri_batch)
                for a in (False, True):
                    _, _, st = run_gpu(ds, rays, any_hit=a, stats=True)
                    assert np.array_equal(st, counts[a]), (variant, tri_batch, a, st, counts[a])
        assert lib.imbart_scene_error_count(ds.handle) == 0
        ds.close()
    finally:
        S.trace_config_restore(saved)


@pytest.mark.gpu
def test_autotuner_chooses_node_width(cuda):
    """GpuScene.autotune_node_width prepares the scene at widths 8 and 4, tunes each query class
    at each, keeps the faster width with its tuned kernels, and the kept scene's hits are the
    oracle's."""
    import torch
    from imbatracer_b200.integrators import GpuScene
    saved = S.trace_config_snapshot()
    try:
        desc = H.scene_desc("config1")
        gs = GpuScene(desc, td=H.traversal_data("config1"))
        dev = torch.device("cuda:0")
        rays = H.ray_set("config1", 50000, seed=31)
        d_rays = torch.from_numpy(np.ascontiguousarray(rays).view(np.float32).reshape(-1, 8)).to(dev)
        assert d_rays.shape[0] == len(rays)
        ray_sets = [(d_rays, torch.zeros((len(rays), 4), dtype=torch.int32, device=dev), f)
                    for f in (N.TRACE_CLOSEST, N.TRACE_ANY)]
        # A byte view of the rays is refused on the host (its first dimension is not the count).
        with pytest.raises(N.ImbartError):
            gs.trace_scene.autotune(to_dev(rays, torch, dev), ray_sets[0][1], N.TRACE_CLOSEST)
        out = gs.autotune_node_width(ray_sets)
        assert out["node_width"] in (4, 8) and set(out["ms"]) == {4, 8}
        assert out["ms"][out["node_width"]] == min(out["ms"].values())
        assert gs.trace_scene.node_width == out["node_width"]
        hits, _, _ = run_gpu(gs.trace_scene, rays)
        assert H.hits_equal(O.trace_node2(H.traversal_data("config1"), rays), hits).all()
        gs.close()
    finally:
        S.trace_config_restore(saved)


@pytest.mark.skipif(not __import__("oracle.refwrap", fromlist=["x"]).imbart_linked_available(),
                    reason="oracle/_ref/libref_imbart.so not built (reference tree absent)")
@pytest.mark.parametrize("name,w,h,spp,max_len", [("mixed", 96, 64, 4, 6), ("config1", 64, 64, 2, 5)])
def test_reference_path_tracer_on_libimbart_traversal(cuda, name, w, h, spp, max_len):
    """The traversal boundary end to end: the reference's own Scene, PathTracer, TileScheduler
    and RayQueue — whose traverse_gpu / traverse_occluded_gpu copy the rays into device
    arrays, call intersect_gpu_masked_instanced / occluded_gpu_masked_instanced and copy the
    hits back (ray_queue.h:269-293, 319-343) — compiled against include/traversal_gpu.h and
    linked to libimbart (oracle/_ref/libref_imbart.so, AnyDSL device arrays in GPU memory)
    render the same image, bit for bit, as the same code over the oracle's traversal."""
    from oracle import refwrap as R
    from tests.test_pt import small_mixed_scene
    d = small_mixed_scene() if name == "mixed" else H.scene_desc(name)
    seed = 4242
    oracle_img = R.RefScene(d).render_pt(w, h, spp, max_len, seed)
    N.load().imbart_invalidate_scenes()       # device arrays of earlier scenes may be reused
    with R.imbart_linked():
        rs = R.RefScene(d)
    img = rs.render_pt(w, h, spp, max_len, seed)
    rs.close()
    N.load().imbart_invalidate_scenes()
    assert oracle_img.sum() > 0
    assert np.array_equal(img.view(np.int32), oracle_img.view(np.int32))
