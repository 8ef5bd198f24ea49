"""The GPU scene builder (imbart_scene_build_gpu): PLOC clustering and a collapse into the
8-wide layout on the device.

A BVH changes which nodes a ray visits, never which triangle it hits: closest hits over
the GPU-built scenes must equal brute force bit for bit (ids, t, u, v), any-hit occlusion
must agree, renders must equal the host-built scene's (float accumulation order aside),
and two builds of the same scene must write identical arrays.
"""
import numpy as np
import pytest

from imbatracer_b200 import native as N
from imbatracer_b200 import scene as S
from imbatracer_b200 import scenegen as G
from oracle import oracle as O
from tests import helpers as H
from tests.test_pt import small_mixed_scene


def scenes():
    return {"tiny": H.scene_desc("tiny"), "config1": H.scene_desc("config1"), "config2": H.scene_desc("config2"),
            "mixed": small_mixed_scene()}


def trace(ds, rays, any_hit=False):
    import torch
    r = torch.from_numpy(rays.view(np.float32).reshape(-1, 8).copy()).cuda()
    h = torch.zeros((len(rays), 4), dtype=torch.int32, device="cuda")
    v = torch.zeros(len(rays), dtype=torch.float32, device="cuda")
    ds.trace(r, h, any_hit=any_hit, v_out=v)
    torch.cuda.synchronize()
    hits = np.zeros(len(rays), N.HIT_DTYPE)
    hits.view(np.int32).reshape(-1, 4)[:] = h.cpu().numpy()
    return hits, v.cpu().numpy()


def mixed_rays(desc, n, seed):
    from imbatracer_b200 import scenegen as G
    lo, hi = G.scene_box(desc)
    return G.random_rays(np.random.default_rng(seed), n, lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "config1", "config2", "mixed"])
def test_gpu_built_scene_hits_equal_brute_force(cuda, name):
    d = scenes()[name]
    ds = S.DeviceScene.build_gpu(d.meshes, d.instances)
    rays = mixed_rays(d, 4000, 11) if name == "mixed" else H.ray_set(name, 4000 if name != "config2" else 1500, seed=7)
    tri_layout = np.concatenate([[0], np.cumsum([m.triangle_count for m in d.meshes])[:-1]]).astype(np.int32)
    hb, vb = O.trace_brute(d.meshes, d.instances, tri_layout, rays, with_v=True)
    hg, vg = trace(ds, rays)
    assert (hb["tri_id"] >= 0).sum() > 0
    assert H.hits_equal(hb, hg).all()
    assert np.array_equal(vb.view(np.int32), vg.view(np.int32))
    ha = O.trace_brute(d.meshes, d.instances, tri_layout, rays, any_hit=True)
    hga, _ = trace(ds, rays, any_hit=True)
    assert np.array_equal(ha["tri_id"] >= 0, hga["tri_id"] >= 0)
    info = ds.info
    assert info.triangles == sum(m.triangle_count for m in d.meshes)
    assert info.instances == len(d.instances) and 0 < info.top_nodes < info.wide_nodes
    ds.close()


class _DeviceBytes:
    """A device byte range as a CUDA array (for torch.as_tensor)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def device_bytes(ptr, n):
    import torch
    return torch.as_tensor(_DeviceBytes(ptr, n), device="cuda").cpu().numpy().tobytes()


@pytest.mark.gpu
def test_gpu_build_is_deterministic(cuda):
    d = scenes()["config2"]
    a = S.DeviceScene.build_gpu(d.meshes, d.instances)
    b = S.DeviceScene.build_gpu(d.meshes, d.instances)
    assert (a.info.wide_nodes, a.info.triangles, a.info.root) == (b.info.wide_nodes, b.info.triangles, b.info.root)
    sizes = (a.info.wide_nodes * 80, a.info.triangles * 48, a.info.instances * 64)
    for pa, pb, n in zip(a.device_arrays(), b.device_arrays(), sizes):
        assert device_bytes(pa, n) == device_bytes(pb, n)


@pytest.mark.gpu
def test_path_traced_frame_on_a_gpu_built_scene(cuda):
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = small_mixed_scene()
    a = PathTracer(GpuScene(d), max_path_len=6).render(4, 99, 64, 48).cpu().numpy()
    b = PathTracer(GpuScene(d, gpu_build=True), max_path_len=6).render(4, 99, 64, 48).cpu().numpy()
    den = np.sqrt(np.mean(a.astype(np.float64) ** 2))
    assert a.sum() > 0 and np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / den <= 1e-5


@pytest.mark.gpu
def test_gpu_build_rejects_bad_input(cuda):
    from imbatracer_b200.scene import Instance, Mesh
    m = Mesh(np.eye(3, dtype=np.float32), np.array([[0, 1, 2, 0]], np.int32))
    m.indices[0, 2] = 5                        # vertex index out of range
    with pytest.raises(N.ImbartError):
        S.DeviceScene.build_gpu([m], [Instance(0)])
    m2 = Mesh(np.eye(3, dtype=np.float32), np.array([[0, 1, 2, 0]], np.int32))
    with pytest.raises(N.ImbartError):
        S.DeviceScene.build_gpu([m2], [Instance(1)])
    N.load().imbart_clear_error()


def _moved(desc, seed):
    """The scene's meshes with every vertex moved: scaled about its mesh's centre by 1.2 and
    jittered (the triangles keep their vertex indices)."""
    rng = np.random.default_rng(seed)
    out = []
    for m in desc.meshes:
        c = m.vertices.mean(0)
        v = (c + (m.vertices - c) * 1.2 + rng.normal(scale=0.01, size=m.vertices.shape)).astype(np.float32)
        out.append(S.Mesh(v, m.indices, m.normals, m.texcoords, m.geom_normals))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name,gpu_built", [("mixed", False), ("mixed", True), ("config1", False),
                                            ("config2", True)])
def test_refit_traces_the_moved_triangles_exactly(cuda, name, gpu_built):
    """imbart_scene_refit after every vertex moved (scaled by 1.2 about each mesh's centre and
    jittered): closest hits equal brute force over the moved triangles bit for bit and
    occlusion equals it, on trees built by the host (SBVH) and on the GPU."""
    from tests.test_pt import small_mixed_scene
    desc = small_mixed_scene() if name == "mixed" else H.scene_desc(name)
    td = S.build_traversal_data(desc.meshes, desc.instances)
    ds = S.DeviceScene.build_gpu(desc.meshes, desc.instances) if gpu_built else S.DeviceScene(td)
    moved = _moved(desc, 7)
    ds.refit(moved)
    lo, hi = G.scene_box(desc)
    ext = hi - lo
    rays = G.random_rays(np.random.default_rng(8), 30000, lo - 0.2 * ext, hi + 0.2 * ext)
    ref = O.trace_brute(moved, desc.instances, td.tri_layout, rays)
    assert (ref["tri_id"] >= 0).sum() > 2000
    from tests.test_traversal_gpu import run_gpu
    hits, _, _ = run_gpu(ds, rays)
    assert H.hits_equal(ref, hits).all(), int((~H.hits_equal(ref, hits)).sum())
    occ, _, _ = run_gpu(ds, rays, any_hit=True)
    assert np.array_equal(occ["tri_id"] >= 0, ref["tri_id"] >= 0)
    # Refitting back to the original positions restores the original hits.
    ds.refit(desc.meshes)
    hits, _, _ = run_gpu(ds, rays)
    assert H.hits_equal(O.trace_node2(td, rays), hits).all()
    ds.close()


@pytest.mark.gpu
def test_refit_rejects_bad_input(cuda):
    import torch
    desc = H.scene_desc("tiny")
    ds = S.DeviceScene(H.traversal_data("tiny"))
    lib = N.load()
    v = torch.zeros((10, 3), dtype=torch.float32, device="cuda")
    t = torch.full((3, 4), 99, dtype=torch.int32, device="cuda")       # vertex 99 of 10
    assert lib.imbart_scene_refit(ds.handle, N.ptr(v), 10, N.ptr(t), 3, None) != 0
    assert lib.imbart_scene_refit(ds.handle, N.ptr(v), 10, N.ptr(t), 0, None) != 0
    lib.imbart_clear_error()
    ds.close()
