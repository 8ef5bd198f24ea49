"""Acceleration cache files (.bvh) as the reference writes and reads them (load_bvh.cpp).

Pinned against the reference itself: files written by the reference's Scene (its own
store_accel_gpu / store_accel_cpu while building) load here into exactly the arrays the
reference loads from them, files written here load in the reference unchanged, and a
scene whose meshes come from files traces like a built one. Malformed files are errors.
"""
import ctypes as C
import os

import numpy as np
import pytest

from imbatracer_b200 import native as N
from imbatracer_b200 import scene as S
from imbatracer_b200 import scenegen as G
from oracle import oracle as O
from oracle import refwrap as R
from tests import helpers as H
from tests.test_pt import small_mixed_scene

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference tree absent)")


def load_all(files, tri_layout, cpu=False):
    """Our loader, mesh after mesh into one pair of arrays (as Scene::build_mesh_accels)."""
    lib = N.load()
    counts = [S.accel_file_counts(f, N.ACCEL_CPU if cpu else N.ACCEL_GPU) for f in files]
    nodes = np.zeros(sum(c[0] for c in counts), N.NODE4_DTYPE if cpu else N.NODE2_DTYPE)
    tris = np.zeros((sum(c[1] for c in counts), 4), np.float32)
    nn, nt = C.c_int(0), C.c_int(0)
    fn = lib.imbart_load_accel_node4 if cpu else lib.imbart_load_accel_node2
    for f, off in zip(files, tri_layout):
        N.check(fn(os.fsencode(f), off, N.ptr(nodes), len(nodes), C.byref(nn), N.ptr(tris), len(tris), C.byref(nt)),
                "load")
    assert nn.value == len(nodes) and nt.value == len(tris)
    return nodes, tris


def tri_layout_of(desc):
    out, off = [], 0
    for m in desc.meshes:
        out.append(off)
        off += m.triangle_count
    return out


@needs_ref
@pytest.mark.parametrize("name", ["mixed", "tiny"])
def test_reference_written_files_load_to_the_reference_arrays(tmp_path, name):
    desc = small_mixed_scene() if name == "mixed" else H.scene_desc("tiny")
    files = [str(tmp_path / f"mesh{i}.bvh") for i in range(len(desc.meshes))]
    R.RefScene(desc, accel_files=files)                 # builds and stores (scene.cpp:62-68)
    assert all(os.path.exists(f) for f in files)
    ref = R.RefScene(desc, accel_files=files)           # loads (scene.cpp:56)
    _, ref_nodes, _, ref_tris = ref.gpu_layout()
    nodes, tris = load_all(files, tri_layout_of(desc))
    assert nodes.tobytes() == ref_nodes[: len(nodes)].tobytes()
    assert np.array_equal(tris.view(np.int32), ref_tris[: len(tris)].view(np.int32))
    # The same arrays through the reference's loader called directly.
    pre_n, pre_t = np.zeros(0, N.NODE2_DTYPE), np.zeros((0, 4), np.float32)
    for f, off in zip(files, tri_layout_of(desc)):
        pre_n, pre_t = R.load_accel(f, off, pre_n, pre_t)
    assert pre_n.tobytes() == nodes.tobytes() and pre_t.tobytes() == tris.tobytes()


@needs_ref
def test_reference_cpu_blocks_load_to_the_reference_arrays(tmp_path):
    desc = small_mixed_scene()
    files = [str(tmp_path / f"mesh{i}.bvh") for i in range(len(desc.meshes))]
    R.RefScene(desc, cpu_buffers=True, accel_files=files)
    for f in files:   # one file, both blocks (the CPU block was written first)
        assert S.accel_file_counts(f, N.ACCEL_CPU) is not None and S.accel_file_counts(f, N.ACCEL_GPU) is not None
    ref = R.RefScene(desc, cpu_buffers=True, accel_files=files)
    _, ref_nodes, _, ref_tris = ref.cpu_layout()
    nodes, tris = load_all(files, tri_layout_of(desc), cpu=True)
    assert nodes.tobytes() == ref_nodes[: len(nodes)].tobytes()
    assert np.array_equal(tris.view(np.int32), ref_tris[: len(tris)].view(np.int32))


@needs_ref
def test_files_written_here_load_in_the_reference(tmp_path):
    desc = small_mixed_scene()
    files = [str(tmp_path / f"own{i}.bvh") for i in range(len(desc.meshes))]
    td = S.build_traversal_data(desc.meshes, desc.instances, accel_files=files)
    n_bottom = td.layout[-1] + S.accel_file_counts(files[-1])[0]
    pre_n, pre_t = np.zeros(0, N.NODE2_DTYPE), np.zeros((0, 4), np.float32)
    for f, off in zip(files, td.tri_layout):
        pre_n, pre_t = R.load_accel(f, off, pre_n, pre_t)
    assert pre_n.tobytes() == td.nodes[:n_bottom].tobytes()
    assert pre_t.tobytes() == td.tris.tobytes()
    # The reference's Scene loads them and its layout traces like ours.
    ref = R.RefScene(desc, accel_files=files)
    root, nodes, insts, tris = ref.gpu_layout()
    assert nodes[:n_bottom].tobytes() == td.nodes[:n_bottom].tobytes()
    # Its top level over our instance transforms (the reference inverts the instance matrices
    # in its own float arithmetic, which moves t and u by ulps).
    ours = {int(i["id"]): i["transf"] for i in td.instances}
    insts = insts.copy()
    for k in range(len(insts)):
        insts[k]["transf"] = ours[int(insts[k]["id"])]
    td_ref = S.TraversalData(root, nodes, insts, tris, td.indices, td.texcoords, td.masks, td.mask_buffer, None,
                             td.tri_layout)
    lo, hi = G.scene_box(desc)
    rays = G.random_rays(np.random.default_rng(5), 4000, lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo))
    hits = O.trace_node2(td, rays)
    assert (hits["tri_id"] >= 0).sum() > 500
    assert H.hits_equal(hits, O.trace_node2(td_ref, rays)).all()


def test_loaded_scene_equals_built_scene_and_traces_exactly(tmp_path):
    desc = H.scene_desc("config1")
    files = [str(tmp_path / f"c1_{i}.bvh") for i in range(len(desc.meshes))]
    built = S.build_traversal_data(desc.meshes, desc.instances, accel_files=files)
    loaded = S.build_traversal_data(desc.meshes, desc.instances, accel_files=files)
    assert built.nodes.tobytes() == loaded.nodes.tobytes() and built.tris.tobytes() == loaded.tris.tobytes()
    rays = H.ray_set("config1", 2000, seed=9)
    hb = O.trace_brute(desc.meshes, desc.instances, loaded.tri_layout, rays)
    assert H.hits_equal(hb, O.trace_node2(loaded, rays)).all()
    wn, wt, wi, root = H.wide_arrays(loaded)
    hw, _, _ = O.wide_walk(wn, wt, wi, root, rays)
    assert H.hits_equal(hb, hw).all()


def test_single_leaf_mesh_loaded_at_another_offset(tmp_path):
    """A one-triangle mesh's BVH is the reference's single-leaf wrapper; read back at another
    node offset than it was written at, its marker stays a marker and the scene converts."""
    d = H.scene_desc("tiny")
    files = [str(tmp_path / "a.bvh"), str(tmp_path / "b.bvh")]
    S.build_traversal_data(d.meshes, d.instances, accel_files=files)
    # Load mesh 1 first (offset 0), then mesh 0 behind it.
    lib = N.load()
    nodes = np.zeros(64, N.NODE2_DTYPE)
    tris = np.zeros((64, 4), np.float32)
    nn, nt = C.c_int(0), C.c_int(0)
    for f in (files[1], files[1], files[0]):
        N.check(lib.imbart_load_accel_node2(os.fsencode(f), 0, N.ptr(nodes), 64, C.byref(nn), N.ptr(tris), 64,
                                            C.byref(nt)), "load")
    assert nodes["right"][0] == 0x76543210 and nodes["right"][1] == 0x76543210
    assert nodes["left"][1] == ~3     # the second copy's leaf follows the first copy's 3 Vec4s


def test_malformed_files_are_errors(tmp_path):
    d = H.scene_desc("tiny")
    good = str(tmp_path / "good.bvh")
    S.build_traversal_data(d.meshes[:1], [d.instances[0]], accel_files=[good])
    data = open(good, "rb").read()
    lib = N.load()
    nodes = np.zeros(64, N.NODE2_DTYPE)
    tris = np.zeros((64, 4), np.float32)

    def load(path):
        nn, nt = C.c_int(0), C.c_int(0)
        rc = lib.imbart_load_accel_node2(os.fsencode(path), 0, N.ptr(nodes), 64, C.byref(nn), N.ptr(tris), 64,
                                         C.byref(nt))
        lib.imbart_clear_error()
        return rc

    assert load(good) == 0
    bad = str(tmp_path / "bad.bvh")
    cases = [b"", b"\x00\x00\x00\x00" + data[4:], data[:3]]
    cases += [data[:k] for k in range(4, len(data), max(1, len(data) // 40))]
    lying = bytearray(data)
    lying[4:12] = (1 << 40).to_bytes(8, "little")          # block size beyond the file
    cases.append(bytes(lying))
    counts = bytearray(data)
    counts[16:20] = (1 << 30).to_bytes(4, "little")        # node count beyond the block
    cases.append(bytes(counts))
    for blob in cases:
        with open(bad, "wb") as f:
            f.write(blob)
        assert load(bad) != 0, len(blob)
    assert load(str(tmp_path / "missing.bvh")) == 1
    # A capacity too small is an error before anything is written.
    nn, nt = C.c_int(0), C.c_int(0)
    n_good = S.accel_file_counts(good)[0]
    assert lib.imbart_load_accel_node2(os.fsencode(good), 0, N.ptr(nodes), n_good - 1, C.byref(nn), N.ptr(tris), 64,
                                       C.byref(nt)) == 6 and nn.value == 0
    lib.imbart_clear_error()
    # A second two-wide block is refused; the CPU block is absent.
    assert lib.imbart_store_accel_node2(os.fsencode(good), N.ptr(nodes), 0, 1, N.ptr(tris), 0, 3, 0) != 0
    lib.imbart_clear_error()
    assert S.accel_file_counts(good, N.ACCEL_CPU) is None


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", ["mixed", "config1"])
def test_reference_written_files_trace_on_the_gpu(cuda, tmp_path, name):
    """Bottom levels loaded from .bvh files the reference's Scene wrote while building
    (store_accel_gpu, scene.cpp:62-68), converted to the 8-wide layout and traced by the GPU
    kernels: closest hits (triangle, instance, t, u, v) bit-exact with the oracle's walk of the
    same arrays, any-hit occlusion equal."""
    from tests.test_traversal_gpu import run_gpu
    desc = small_mixed_scene() if name == "mixed" else H.scene_desc(name)
    files = [str(tmp_path / f"{name}{i}.bvh") for i in range(len(desc.meshes))]
    R.RefScene(desc, accel_files=files)                  # the reference builds and stores
    assert all(os.path.exists(f) for f in files)
    td = S.build_traversal_data(desc.meshes, desc.instances, accel_files=files)
    _, ref_nodes, _, _ = R.RefScene(desc, accel_files=files).gpu_layout()
    n_bottom = td.layout[-1] + S.accel_file_counts(files[-1])[0]
    assert td.nodes[:n_bottom].tobytes() == ref_nodes[:n_bottom].tobytes()   # loaded, not rebuilt
    lo, hi = G.scene_box(desc)
    rays = G.random_rays(np.random.default_rng(11), 50000, lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo))
    ds = S.DeviceScene(td)
    ref, ref_v = O.trace_node2(td, rays, with_v=True)
    hits, v, _ = run_gpu(ds, rays)
    assert (ref["tri_id"] >= 0).sum() > 1000
    assert H.hits_equal(ref, hits).all()
    assert np.array_equal(ref_v.view(np.int32), v.view(np.int32))
    occ, _, _ = run_gpu(ds, rays, any_hit=True)
    assert np.array_equal(occ["tri_id"] >= 0, O.trace_node2(td, rays, any_hit=True)["tri_id"] >= 0)
    ds.close()
