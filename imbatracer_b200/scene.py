"""Host-side scene: meshes, instances, materials and lights, and the traversal data.

Mirrors the reference's Scene (src/imbatracer/render/scene.{h,cpp}): per-mesh bottom-level BVHs
are laid out one after another in one node array (scene.cpp:37-72), global triangle ids are
offset per mesh (tri_layout, scene.cpp:75-97), the top-level BVH follows at node index
`node_count` which becomes the root (scene.cpp:103-117, 167-188). The BVHs are written by
libimbart's binned-SAH builder in the reference two-wide GPU layout, then converted by
libimbart into the compressed 8-wide layout resident on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field

import numpy as np

from . import native as N


@dataclass
class Mesh:
    """Triangle mesh: vertices (V,3), indices (T,4) = {i0, i1, i2, material} (mesh.h:103-114),
    optional per-vertex normals (V,3) and texture coordinates (V,2)."""
    vertices: np.ndarray
    indices: np.ndarray
    normals: np.ndarray | None = None
    texcoords: np.ndarray | None = None
    geom_normals: np.ndarray | None = None

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.int32).reshape(-1, 4)
        if self.texcoords is None:
            self.texcoords = np.zeros((len(self.vertices), 2), np.float32)
        self.texcoords = np.ascontiguousarray(self.texcoords, dtype=np.float32).reshape(-1, 2)
        if self.geom_normals is None:
            self.geom_normals = face_normals(self.vertices, self.indices)
        if self.normals is None:
            self.normals = vertex_normals(self.vertices, self.indices, self.geom_normals)
        self.normals = np.ascontiguousarray(self.normals, dtype=np.float32).reshape(-1, 3)

    @property
    def triangle_count(self) -> int:
        return len(self.indices)

    def bounding_box(self) -> tuple[np.ndarray, np.ndarray]:
        return self.vertices.min(0), self.vertices.max(0)


def face_normals(v: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Normalized geometric normals cross(v1 - v0, v2 - v0) per face (mesh.cpp)."""
    a, b, c = v[idx[:, 0]], v[idx[:, 1]], v[idx[:, 2]]
    n = np.cross(b - a, c - a)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    ln[ln == 0] = 1.0
    return (n / ln).astype(np.float32)


def vertex_normals(v: np.ndarray, idx: np.ndarray, fn: np.ndarray) -> np.ndarray:
    """Area-unweighted average of adjacent face normals, normalized."""
    acc = np.zeros_like(v, dtype=np.float64)
    for k in range(3):
        np.add.at(acc, idx[:, k], fn)
    ln = np.linalg.norm(acc, axis=1, keepdims=True)
    ln[ln == 0] = 1.0
    return (acc / ln).astype(np.float32)


def _cofactor_terms():
    """For each entry (i, j) of the adjugate of a 4x4 matrix: its sign and six products of
    three entries, in the order the reference's invert (float4x4.h:144-197) sums them. With
    the rows R = (r0, r1, r2) other than j and the columns C = (c0, c1, c2) other than i, the
    products are (r0,c0)(r1,c1)(r2,c2), (r0,c0)(r1,c2)(r2,c1), (r1,c0)(r0,c1)(r2,c2),
    (r1,c0)(r0,c2)(r2,c1), (r2,c0)(r0,c1)(r1,c2), (r2,c0)(r0,c2)(r1,c1) with the signs
    + - - + + -, all negated when i + j is odd."""
    pattern = [((0, 0), (1, 1), (2, 2), 1), ((0, 0), (1, 2), (2, 1), -1), ((1, 0), (0, 1), (2, 2), -1),
               ((1, 0), (0, 2), (2, 1), 1), ((2, 0), (0, 1), (1, 2), 1), ((2, 0), (0, 2), (1, 1), -1)]
    table = {}
    for i in range(4):
        for j in range(4):
            rows = [r for r in range(4) if r != j]
            cols = [c for c in range(4) if c != i]
            sgn = 1 if (i + j) % 2 == 0 else -1
            table[i, j] = [(sgn * s, (rows[a[0]], cols[a[1]]), (rows[b[0]], cols[b[1]]), (rows[c[0]], cols[c[1]]))
                           for a, b, c, s in pattern]
    return table


_COFACTORS = _cofactor_terms()


def invert_f32(m: np.ndarray) -> np.ndarray:
    """Inverse of a 4x4 matrix in single precision with the reference's operation order
    (float4x4.h:144-197: adjugate by cofactors summed left to right, each product formed left
    to right, det = a[0] . column 0 of the adjugate, then every entry times the rounded 1/det;
    a singular matrix gives zeros), so instance transforms, hits and shading normals agree
    with the reference's bit for bit."""
    a = np.asarray(m, np.float32).reshape(4, 4)
    f = np.float32
    res = np.zeros((4, 4), np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        for (i, j), terms in _COFACTORS.items():
            acc = None
            for s, (r0, c0), (r1, c1), (r2, c2) in terms:
                prod = f(f(a[r0, c0] * a[r1, c1]) * a[r2, c2])
                if acc is None:
                    acc = prod if s > 0 else f(-prod)
                else:
                    acc = f(acc + prod) if s > 0 else f(acc - prod)
            res[i, j] = acc
        det = f(f(f(f(a[0, 0] * res[0, 0]) + f(a[0, 1] * res[1, 0])) + f(a[0, 2] * res[2, 0])) + f(a[0, 3] * res[3, 0]))
        if det == 0:
            return np.zeros((4, 4), np.float32)
        return (res * f(f(1.0) / det)).astype(np.float32)


@dataclass
class Instance:
    """A mesh instance with its object-to-world matrix and the world-to-object inverse the
    reference stores beside it (mesh.h:19-27, computed as float4x4.h's invert does)."""
    mesh_id: int
    mat: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))

    def __post_init__(self):
        self.mat = np.asarray(self.mat, np.float32).reshape(4, 4)
        self.inv_mat = invert_f32(self.mat)[:3].copy()


class TraversalData:
    """The reference-layout traversal arrays of a scene (ray_queue.h:42-54)."""

    def __init__(self, root, nodes, instances, tris, indices, texcoords, masks, mask_buffer, layout, tri_layout):
        self.root = root
        self.nodes = nodes
        self.instances = instances
        self.tris = tris
        self.indices = indices
        self.texcoords = texcoords
        self.masks = masks
        self.mask_buffer = mask_buffer
        self.layout = layout
        self.tri_layout = tri_layout


def accel_file_counts(path: str, block_type: int = N.ACCEL_GPU) -> tuple[int, int] | None:
    """(nodes, Vec4s) of the file's block of `block_type`, or None when it has none or does
    not exist; raises on a malformed file."""
    if not path or not os.path.exists(path):
        return None
    nn, nv = C.c_int(0), C.c_int(0)
    rc = N.load().imbart_accel_file_info(os.fsencode(path), block_type, C.byref(nn), C.byref(nv))
    if rc == -1:
        return None
    N.check(rc, "imbart_accel_file_info")
    return nn.value, nv.value


def build_traversal_data(meshes: list[Mesh], instances: list[Instance], leaf_size: int = 2,
                         masks: np.ndarray | None = None, mask_buffer: np.ndarray | None = None,
                         split_budget: float = 2.0, accel_files: list[str | None] | None = None) -> TraversalData:
    """Builds all bottom-level BVHs and the top-level BVH in the reference two-wide layout.

    The bottom levels use spatial splits (SBVH, as the reference's GPU adapter builds its
    meshes with SplitBvhBuilder), allowing up to split_budget * triangles extra triangle
    references per mesh; 0 builds object splits only. accel_files[i] (optional) is mesh i's
    acceleration cache file, as Scene::build_mesh_accels uses them (scene.cpp:51-68): the
    mesh's BVH is loaded from it when it has a two-wide block, else built and appended to it."""
    lib = N.load()
    files = list(accel_files) if accel_files is not None else [None] * len(meshes)
    assert len(files) == len(meshes)
    cached = [accel_file_counts(f) for f in files]
    node_need = [c[0] if c else int(m.triangle_count * (1.0 + split_budget)) + 1 for m, c in zip(meshes, cached)]
    vec4_need = [c[1] if c else 3 * int(m.triangle_count * (1.0 + split_budget)) for m, c in zip(meshes, cached)]
    node_cap = sum(node_need) + 2 * len(instances) + 1
    nodes = np.zeros(node_cap, N.NODE2_DTYPE)
    tris = np.zeros((sum(vec4_need), 4), np.float32)
    n_nodes = C.c_int(0)
    n_tv = C.c_int(0)
    layout, tri_layout = [], []
    tri_off = 0
    for m, path, c in zip(meshes, files, cached):
        layout.append(n_nodes.value)
        tri_layout.append(tri_off)
        if c is not None:
            N.check(lib.imbart_load_accel_node2(os.fsencode(path), tri_off, N.ptr(nodes), node_cap, C.byref(n_nodes),
                                                N.ptr(tris), len(tris), C.byref(n_tv)), "imbart_load_accel_node2")
            tri_off += m.triangle_count
            continue
        tris_first = n_tv.value
        rc = lib.imbart_build_mesh_node2_ex(N.ptr(m.vertices), len(m.vertices), 3, N.ptr(m.indices),
                                            m.triangle_count, tri_off, leaf_size, split_budget, N.ptr(nodes),
                                            node_cap, C.byref(n_nodes), N.ptr(tris), len(tris), C.byref(n_tv))
        N.check(rc, "imbart_build_mesh_node2_ex")
        if path:
            N.check(lib.imbart_store_accel_node2(os.fsencode(path), N.ptr(nodes), layout[-1], n_nodes.value,
                                                 N.ptr(tris), tris_first, n_tv.value, tri_off),
                    "imbart_store_accel_node2")
        tri_off += m.triangle_count
    node_count = n_nodes.value
    # Instance world boxes. The reference transforms the mesh box (centre +- |M| * half extent,
    # gpu_adapter.cpp:171-179), which for rotated instances is up to sqrt(3) times wider per
    # axis than the instance itself; here the box is the bound of the transformed vertices
    # (of their convex hull for large meshes, which has the same bound), rounded outward.
    boxes = np.zeros((len(instances), 6), np.float32)
    inv = np.zeros((len(instances), 12), np.float32)
    roots = np.zeros(len(instances), np.int32)
    hull = [m.vertices.astype(np.float64) for m in meshes]
    for i, inst in enumerate(instances):
        w = hull[inst.mesh_id] @ inst.mat[:3, :3].astype(np.float64).T + inst.mat[:3, 3].astype(np.float64)
        lo, hi = w.min(0), w.max(0)
        pad = 1e-6 * (np.abs(lo).max() + np.abs(hi).max() + (hi - lo).max())
        boxes[i, :3] = np.nextafter((lo - pad).astype(np.float32), np.float32(-np.inf))
        boxes[i, 3:] = np.nextafter((hi + pad).astype(np.float32), np.float32(np.inf))
        inv[i] = inst.inv_mat.reshape(-1)
        roots[i] = layout[inst.mesh_id]
    insts = np.zeros(len(instances), N.INST_DTYPE)
    rc = lib.imbart_build_top_node2(N.ptr(boxes), N.ptr(inv), N.ptr(roots), len(instances), N.ptr(nodes),
                                    node_cap, C.byref(n_nodes), N.ptr(insts))
    N.check(rc, "imbart_build_top_node2")
    nodes = nodes[: n_nodes.value].copy()
    tris = tris[: n_tv.value].copy()
    # Global index and texcoord buffers (scene.cpp:75-97): texcoord indices offset per mesh.
    idx_parts, tc_parts = [], []
    tc_off = 0
    for m in meshes:
        ii = m.indices.copy()
        ii[:, :3] += tc_off
        idx_parts.append(ii.reshape(-1))
        tc_parts.append(m.texcoords)
        tc_off += len(m.texcoords)
    indices = np.ascontiguousarray(np.concatenate(idx_parts).astype(np.int32))
    texcoords = np.ascontiguousarray(np.concatenate(tc_parts).astype(np.float32))
    if masks is None:
        n_mats = int(max(m.indices[:, 3].max() for m in meshes)) + 1
        masks = np.zeros(n_mats, N.MASK_DTYPE)
        masks["width"] = 1
        masks["height"] = 1
        mask_buffer = np.ones(4, np.uint8)  # MaskBuffer starts with 4 opaque texels (mask.h:24-28)
    return TraversalData(node_count, nodes, insts, tris, indices, texcoords, masks,
                         np.ascontiguousarray(mask_buffer, dtype=np.uint8), layout, tri_layout)


def build_descs(meshes: list[Mesh], instances: list[Instance]):
    """Mesh and instance descriptors of imbart_scene_build_gpu (triangles numbered mesh after
    mesh); returns (meshes, instances, arrays to keep alive during the call)."""
    md = (N.MeshDesc * len(meshes))()
    keep, off = [], 0
    for k, m in enumerate(meshes):
        v = np.ascontiguousarray(m.vertices, np.float32)
        ix = np.ascontiguousarray(m.indices, np.int32)
        keep += [v, ix]
        md[k].vertices, md[k].n_vertices = N.ptr(v), len(v)
        md[k].indices, md[k].n_tris = N.ptr(ix), len(ix)
        md[k].tri_offset = off
        off += m.triangle_count
    idesc = (N.InstanceDesc * len(instances))()
    for i, inst in enumerate(instances):
        idesc[i].obj_to_world[:] = [float(x) for x in inst.mat[:3].reshape(-1)]
        idesc[i].world_to_obj[:] = [float(x) for x in inst.inv_mat.reshape(-1)]
        idesc[i].mesh = inst.mesh_id
        idesc[i].id = i
    return md, idesc, keep


def _nbytes(t) -> int:
    return int(t.numel() * t.element_size()) if hasattr(t, "element_size") else int(t.nbytes)


def _check_ray_buffers(rays, hits, n: int, what: str) -> None:
    """Rays are 32 B and hits 16 B records: the buffers must hold n of each."""
    if n < 0 or _nbytes(rays) < 32 * n or _nbytes(hits) < 16 * n:
        raise N.ImbartError(f"{what}: {n} rays need {32 * n} B of rays and {16 * n} B of hits "
                            f"(have {_nbytes(rays)} and {_nbytes(hits)})")


# The node width is a process setting of the library; DeviceScene(node_width=...) changes it
# only for its own conversion, under this lock.
_NODE_WIDTH_LOCK = threading.Lock()

TRACE_CLASSES = (N.TRACE_CLOSEST | N.TRACE_COHERENT, N.TRACE_CLOSEST, N.TRACE_ANY)


def trace_config_snapshot() -> list[tuple[int, int, int, int]]:
    """The process-wide kernel configuration of the three query classes:
    (flags, variant, refill lanes, triangle batch) each."""
    lib = N.load()
    out = []
    for flags in TRACE_CLASSES:
        v, r = C.c_int(0), C.c_int(0)
        N.check(lib.imbart_get_trace_class(flags, C.byref(v), C.byref(r)), "imbart_get_trace_class")
        out.append((flags, v.value, r.value, lib.imbart_get_trace_tri_batch(flags)))
    return out


def trace_config_restore(snapshot) -> None:
    lib = N.load()
    for flags, v, r, b in snapshot:
        N.check(lib.imbart_set_trace_class(flags, v, r), "imbart_set_trace_class")
        N.check(lib.imbart_set_trace_tri_batch(flags, b), "imbart_set_trace_tri_batch")


class DeviceScene:
    """A prepared scene resident on one GPU (imbart_scene)."""

    @classmethod
    def build_gpu(cls, meshes: list[Mesh], instances: list[Instance], device: int = 0, stream=None) -> "DeviceScene":
        """The scene built on the GPU (imbart_scene_build_gpu) from its meshes and instances;
        triangle ids are numbered mesh after mesh as build_traversal_data numbers them.
        `build_ms` holds the build's wall time."""
        lib = N.load()
        md, idesc, keep = build_descs(meshes, instances)
        ms = C.c_float(0.0)
        st = None if stream is None else stream.cuda_stream
        h = lib.imbart_scene_build_gpu(md, len(meshes), idesc, len(instances), device, st, C.byref(ms))
        if not h:
            code, msg = N.last_error()
            raise N.ImbartError(f"imbart_scene_build_gpu failed ({code}): {msg}")
        self = cls.__new__(cls)
        self.handle, self.device, self.td = h, device, None
        info = N.SceneInfo()
        N.check(lib.imbart_scene_get_info(h, C.byref(info)), "imbart_scene_get_info")
        self.info = info
        self.build_ms = ms.value
        return self

    def __init__(self, td: TraversalData, device: int = 0, node_width: int | None = None):
        """node_width: 8 or 4 for this scene (imbart_set_node_width around the conversion, under
        a lock that Python callers share); None keeps the process setting."""
        lib = N.load()
        with _NODE_WIDTH_LOCK:
            prev_width = lib.imbart_get_node_width()
            if node_width is not None:
                N.check(lib.imbart_set_node_width(node_width), "imbart_set_node_width")
            try:
                h = lib.imbart_scene_from_node2(td.root, N.ptr(td.nodes), len(td.nodes), N.ptr(td.instances),
                                                len(td.instances), N.ptr(td.tris), len(td.tris), N.ptr(td.indices),
                                                len(td.indices), N.ptr(td.texcoords), len(td.texcoords),
                                                N.ptr(td.masks), len(td.masks), N.ptr(td.mask_buffer),
                                                len(td.mask_buffer), device)
            finally:
                lib.imbart_set_node_width(prev_width)
        if not h:
            code, msg = N.last_error()
            raise N.ImbartError(f"imbart_scene_from_node2 failed ({code}): {msg}")
        self.handle = h
        self.device = device
        self.td = td
        info = N.SceneInfo()
        N.check(lib.imbart_scene_get_info(h, C.byref(info)), "imbart_scene_get_info")
        self.info = info

    def trace(self, rays, hits, count: int | None = None, any_hit: bool = False, stream=None, v_out=None):
        """Traces device tensors: rays (N,8) float32, hits (N,4) int32; stream-ordered."""
        lib = N.load()
        n = rays.shape[0] if count is None else count
        _check_ray_buffers(rays, hits, n, "trace")
        st = None if stream is None else stream.cuda_stream
        flags = N.TRACE_ANY if any_hit else N.TRACE_CLOSEST
        if v_out is None:
            rc = lib.imbart_trace(self.handle, N.ptr(rays), N.ptr(hits), n, flags, st)
        else:
            rc = lib.imbart_trace_uv(self.handle, N.ptr(rays), N.ptr(hits), N.ptr(v_out), n, flags, st)
        N.check(rc, "imbart_trace")

    def refit(self, meshes: list[Mesh], stream=None) -> None:
        """imbart_scene_refit with the meshes' new vertex positions (same topology, triangles
        numbered mesh after mesh as the scene was built)."""
        import torch
        dev = torch.device("cuda", self.device)
        verts = np.ascontiguousarray(np.concatenate([m.vertices for m in meshes]).astype(np.float32))
        tv, off = [], 0
        for m in meshes:
            t = np.zeros((m.triangle_count, 4), np.int32)
            t[:, :3] = m.indices[:, :3] + off
            tv.append(t)
            off += len(m.vertices)
        tv = np.concatenate(tv)
        d_v = torch.from_numpy(verts).to(dev)
        d_t = torch.from_numpy(tv).to(dev)
        st = None if stream is None else stream.cuda_stream
        N.check(N.load().imbart_scene_refit(self.handle, N.ptr(d_v), len(verts), N.ptr(d_t), len(tv), st),
                "imbart_scene_refit")

    def trace_host(self, rays: np.ndarray, hits: np.ndarray, any_hit: bool = False, stream=None):
        lib = N.load()
        st = None if stream is None else stream.cuda_stream
        rc = lib.imbart_trace_host(self.handle, N.ptr(rays), N.ptr(hits), len(rays),
                                   N.TRACE_ANY if any_hit else N.TRACE_CLOSEST, st)
        N.check(rc, "imbart_trace_host")

    def autotune(self, rays, hits, flags: int, stream=None) -> dict:
        """imbart_trace_autotune on device tensors: picks the kernel configuration of the query
        class `flags` (TRACE_CLOSEST, TRACE_ANY, TRACE_CLOSEST | TRACE_COHERENT) for these rays."""
        t = N.TraceTuning()
        st = None if stream is None else stream.cuda_stream
        _check_ray_buffers(rays, hits, rays.shape[0], "autotune")
        N.check(N.load().imbart_trace_autotune(self.handle, N.ptr(rays), N.ptr(hits), rays.shape[0], flags, st,
                                               C.byref(t)), "imbart_trace_autotune")
        return {"variant": t.variant, "refill": t.refill, "tri_batch": t.tri_batch, "ms": t.ms,
                "default_ms": t.default_ms}

    @property
    def node_width(self) -> int:
        return int(self.info.node_width)

    def device_arrays(self):
        lib = N.load()
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        N.check(lib.imbart_scene_get_device_arrays(self.handle, C.byref(a), C.byref(b), C.byref(c)), "arrays")
        return a.value, b.value, c.value

    def close(self):
        if self.handle:
            N.load().imbart_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
