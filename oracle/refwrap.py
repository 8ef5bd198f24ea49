"""Python access to oracle/_ref/libref.so — the reference's own C++ built in place from its
sources (oracle/ref/build_ref.py). TEST INFRASTRUCTURE ONLY: used to pin the oracle and to
produce golden outputs; the product never loads it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref.so")

# The same harness built a second time with the reference's traversal entry points taken from
# libimbart instead of the oracle and its AnyDSL device arrays in GPU memory
# (oracle/ref/build_ref.py: libref_imbart.so), for the drop-in test of the traversal boundary.
LIB_IMBART = os.path.join(HERE, "_ref", "libref_imbart.so")

_libs: dict = {}
_active = LIB


def available() -> bool:
    return os.path.exists(LIB)


def imbart_linked_available() -> bool:
    return os.path.exists(LIB_IMBART)


class imbart_linked:
    """Within this context, RefScene objects are created by libref_imbart.so: the reference's
    RayQueue::traverse_gpu / traverse_occluded_gpu (ray_queue.h:269-343) call libimbart's
    intersect_gpu_masked_instanced / occluded_gpu_masked_instanced on device buffers."""

    def __enter__(self):
        global _active
        self.saved, _active = _active, LIB_IMBART
        return self

    def __exit__(self, *exc):
        global _active
        _active = self.saved
        return False


def reference_root() -> str | None:
    """The reference tree libref.so was built from (IMBART_REFERENCE, else the path the build
    recipe recorded), or None where it is absent (for example on a machine that only received
    the built files). Tests read its scene files from copies, never in place, because loading
    a scene with `accel` lines makes the reference write cache files beside it."""
    root = os.environ.get("IMBART_REFERENCE")
    if not root:
        try:
            with open(os.path.join(HERE, "_ref", "reference_root.txt")) as f:
                root = f.read().strip()
        except OSError:
            return None
    return root if root and os.path.isdir(root) else None


def copy_reference_scenes(dst: str, sub: str = "cornell") -> str | None:
    """Copies the reference's test/scenes/<sub> folder (scene, OBJ and MTL files, without cache
    files) to dst/<sub> and returns that folder; None without the reference tree."""
    import shutil
    root = reference_root()
    src = os.path.join(root, "test", "scenes", sub) if root else None
    if not src or not os.path.isdir(src):
        return None
    out = os.path.join(dst, sub)
    shutil.copytree(src, out, ignore=shutil.ignore_patterns("*.bvh"), dirs_exist_ok=True)
    for dirpath, _, files in os.walk(out):      # the copies must be writable: caches go there
        os.chmod(dirpath, 0o755)
        for f in files:
            os.chmod(os.path.join(dirpath, f), 0o644)
    return out


def load() -> C.CDLL:
    _lib = _libs.get(_active)
    if _lib is None:
        lib = C.CDLL(_active)
        P, I, U64, F = C.c_void_p, C.c_int, C.c_uint64, C.c_float
        sig = {
            "imbart_ref_set_seed": (None, [U64, U64]),
            "imbart_ref_set_threads": (None, [I, I]),
            "ref_rng_floats": (None, [U64, I, P]),
            "ref_rng_ints": (None, [U64, I, I, I, P]),
            "ref_camera_rays": (I, [I, I, I, P, P, P, F, U64, P, P, P, P]),
            "ref_hashgrid_query": (I, [P, I, F, P, I, I, P, P]),
            "ref_scene_create": (P, [I, P, P, P, P, P, P, P, I, P, P, I, P, P, I, P, P]),
            "ref_scene_destroy": (None, [P]),
            "ref_scene_extend": (I, [P, I, P, P, I, P, P, P, P]),
            "ref_scene_gpu_layout": (I, [P, C.POINTER(I), C.POINTER(P), C.POINTER(P), C.POINTER(P), P]),
            "ref_scene_bsphere": (None, [P, P]),
            "ref_scene_cpu_layout": (I, [P, C.POINTER(I), C.POINTER(P), C.POINTER(P), C.POINTER(P), P]),
            "ref_set_next_scene_options": (None, [I, I, P]),
            "ref_scene_load": (P, [C.c_char_p, P]),
            "ref_scene_counts": (None, [P, P]),
            "ref_scene_meshes": (None, [P, P, P, P, P, P, P]),
            "ref_scene_instances": (None, [P, P, P]),
            "ref_scene_materials": (I, [P, P, P]),
            "ref_scene_lights": (I, [P, P, P]),
            "ref_scene_textures": (None, [P, P, P]),
            "ref_scene_masks": (None, [P, P, P]),
            "ref_scene_env": (I, [P, P, P, P]),
            "ref_load_accel": (I, [I, C.c_char_p, I, P, I, P, I, P, I, P, P, I, P]),
            "ref_store_accel": (I, [I, C.c_char_p, P, I, I, P, I, I, I]),
            "ref_render_pt": (I, [P, I, I, P, P, P, F, I, I, U64, P]),
            "ref_render_pt_threads": (I, [P, I, I, P, P, P, F, I, I, U64, I, I, P, P]),
            "ref_render_pt_rr": (I, [P, I, I, P, P, P, F, I, I, I, U64, P]),
            "ref_vcm_create": (P, [P, I, I, I, P, P, P, F, I, I, I, I, I, F, I, U64]),
            "ref_vcm_destroy": (None, [P]),
            "ref_vcm_info": (None, [P, P]),
            "ref_vcm_begin_iteration": (F, [P, I, P]),
            "ref_vcm_light_pass": (None, [P, U64, U64, P]),
            "ref_vcm_light_vertices": (I, [P, P, I]),
            "ref_vcm_camera_pass": (None, [P, U64, P]),
            "ref_vcm_time_grid": (None, [P, I, I, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _lib = _libs[_active] = lib
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data


def rng_floats(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    load().ref_rng_floats(seed & (2 ** 64 - 1), n, _p(out))
    return out


def rng_ints(seed: int, n: int, lo: int, hi: int) -> np.ndarray:
    out = np.zeros(n, np.int32)
    load().ref_rng_ints(seed & (2 ** 64 - 1), n, lo, hi, _p(out))
    return out


def camera_rays(w, h, spp, pos, dir, up, fov, seed_base):
    n = w * h * spp
    rays = np.zeros((n, 8), np.float32)
    pid = np.zeros(n, np.int32)
    sid = np.zeros(n, np.int32)
    st = np.zeros(n, np.uint64)
    # Keep the input arrays alive across the call.
    p3, d3, u3 = (np.ascontiguousarray(np.asarray(v, np.float32)) for v in (pos, dir, up))
    rc = load().ref_camera_rays(w, h, spp, _p(p3), _p(d3), _p(u3), fov, seed_base, _p(rays), _p(pid), _p(sid),
                                _p(st))
    assert rc == n
    return rays, pid, sid, st


def hashgrid_query(pos, radius, queries, k):
    pos = np.ascontiguousarray(pos, np.float32)
    q = np.ascontiguousarray(queries, np.float32)
    ids = np.zeros((len(q), k), np.int32)
    cnt = np.zeros(len(q), np.int32)
    load().ref_hashgrid_query(_p(pos), len(pos), radius, _p(q), len(q), k, _p(ids), _p(cnt))
    return ids, cnt


GPU_GRID_LIB = os.path.join(HERE, "_ref", "libref_gpu_grid.so")


def gpu_grid_available() -> bool:
    return os.path.exists(GPU_GRID_LIB)


def light_vertices_merge_gpu(pos, radius, queries, k):
    """The reference's LightVertices with its HashGrid replaced, by include path, by the C++
    adapter over libimbart's GPU grid (oracle/ref/ref_gpu_grid.cpp): cache indices and counts
    of get_merge at each query."""
    lib = C.CDLL(GPU_GRID_LIB)
    fn = lib.refgpu_light_vertices_merge
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    pos = np.ascontiguousarray(pos, np.float32)
    q = np.ascontiguousarray(queries, np.float32)
    ids = np.zeros((len(q), k), np.int32)
    cnt = np.zeros(len(q), np.int32)
    assert fn(_p(pos), len(pos), radius, _p(q), len(q), k, _p(ids), _p(cnt)) == 0
    return ids, cnt


def material_arrays(materials):
    kinds = np.array([m.kind for m in materials], np.int32)
    prm = np.zeros((len(materials), 16), np.float32)
    for i, m in enumerate(materials):
        prm[i, 0:3] = m.color
        prm[i, 3:6] = m.specular
        prm[i, 6] = m.exponent
        prm[i, 7] = m.eta
        prm[i, 8] = m.kappa
        prm[i, 9:12] = m.emission
    return kinds, prm


def load_accel(path, tri_id_offset, pre_nodes, pre_tris, cpu=False):
    """The reference's load_accel_gpu / _cpu appending to copies of pre_nodes / pre_tris;
    None when it returns false."""
    from imbatracer_b200.native import NODE2_DTYPE, NODE4_DTYPE
    dt = NODE4_DTYPE if cpu else NODE2_DTYPE
    pre_nodes = np.ascontiguousarray(pre_nodes, dtype=dt)
    pre_tris = np.ascontiguousarray(pre_tris, dtype=np.float32).reshape(-1, 4)
    cap_n, cap_t = len(pre_nodes) + (1 << 22), len(pre_tris) + (1 << 24)
    nodes = np.zeros(cap_n, dt)
    tris = np.zeros((cap_t, 4), np.float32)
    nn, nt = C.c_int(0), C.c_int(0)
    rc = load().ref_load_accel(1 if cpu else 0, os.fsencode(path), tri_id_offset, _p(pre_nodes), len(pre_nodes),
                               _p(pre_tris), len(pre_tris), _p(nodes), cap_n, C.byref(nn), _p(tris), cap_t,
                               C.byref(nt))
    if rc != 0:
        return None
    return nodes[: nn.value].copy(), tris[: nt.value].copy()


def store_accel(path, nodes, node_offset, tris, tris_offset, tri_id_offset, cpu=False) -> bool:
    """The reference's store_accel_gpu / _cpu."""
    from imbatracer_b200.native import NODE2_DTYPE, NODE4_DTYPE
    nodes = np.ascontiguousarray(nodes, dtype=NODE4_DTYPE if cpu else NODE2_DTYPE)
    tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 4)
    return load().ref_store_accel(1 if cpu else 0, os.fsencode(path), _p(nodes), node_offset, len(nodes), _p(tris),
                                  tris_offset, len(tris), tri_id_offset) == 0


class RefScene:
    """The reference's Scene built from a SceneDesc with the reference's adapters (SBVH
    bottom level, binned top level) into its GPU two-wide layout (and its CPU four-wide
    layout with cpu_buffers). accel_files: per-mesh acceleration cache files, loaded or
    written by the reference's Scene::build_mesh_accels."""

    def __init__(self, desc, cpu_buffers: bool = False, accel_files=None):
        self.desc = desc
        self.lib = load()
        names = None
        if accel_files is not None:
            enc = [os.fsencode(f) if f else None for f in accel_files]
            names = (C.c_char_p * len(enc))(*enc)
        self.lib.ref_set_next_scene_options(1 if cpu_buffers else 0, len(accel_files or []), names)
        meshes = desc.meshes
        nv = np.array([len(m.vertices) for m in meshes], np.int32)
        nt = np.array([m.triangle_count for m in meshes], np.int32)
        verts = np.ascontiguousarray(np.concatenate([m.vertices for m in meshes]).astype(np.float32))
        idx = np.ascontiguousarray(np.concatenate([m.indices.reshape(-1) for m in meshes]).astype(np.int32))
        nrm = np.ascontiguousarray(np.concatenate([m.normals for m in meshes]).astype(np.float32))
        tc = np.ascontiguousarray(np.concatenate([m.texcoords for m in meshes]).astype(np.float32))
        gn = np.ascontiguousarray(np.concatenate([m.geom_normals for m in meshes]).astype(np.float32))
        im = np.array([i.mesh_id for i in desc.instances], np.int32)
        mats = np.ascontiguousarray(np.stack([i.mat.reshape(-1) for i in desc.instances]).astype(np.float32))
        kinds, prm = material_arrays(desc.materials)
        lights = np.zeros((max(len(desc.lights), 1), 12), np.float32)
        for i, (p0, p1, p2, e) in enumerate(desc.lights):
            lights[i] = np.concatenate([p0, p1, p2, e])
        env = None if desc.env_intensity is None else np.array(desc.env_intensity, np.float32)
        self._keep = (nv, nt, verts, idx, nrm, tc, gn, im, mats, kinds, prm, lights, env)
        self.handle = self.lib.ref_scene_create(len(meshes), _p(nv), _p(nt), _p(verts), _p(idx), _p(nrm), _p(tc),
                                              _p(gn), len(im), _p(im), _p(mats), len(kinds), _p(kinds), _p(prm),
                                              len(desc.lights), _p(lights), _p(env))
        assert self.handle
        delta, tex = list(getattr(desc, "delta_lights", [])), list(getattr(desc, "textures", []))
        mtex = np.array([getattr(m, "texture", -1) for m in desc.materials], np.int32)
        mbump = np.array([getattr(m, "bump", -1) for m in desc.materials], np.int32)
        if delta or tex or (mtex >= 0).any() or (mbump >= 0).any():
            kinds = np.array([k for k, _ in delta] or [0], np.int32)
            lp = np.ascontiguousarray(np.array([p for _, p in delta] or [[0.0] * 12], np.float32))
            dims = np.array([[t.shape[1], t.shape[0]] for t in tex] or [[0, 0]], np.int32)
            px = (np.ascontiguousarray(np.concatenate([np.asarray(t, np.float32).reshape(-1) for t in tex]))
                  if tex else np.zeros(4, np.float32))
            self._keep2 = (kinds, lp, dims, px, mtex, mbump)
            rc = self.lib.ref_scene_extend(self.handle, len(delta), _p(kinds), _p(lp), len(tex), _p(dims), _p(px),
                                         _p(mtex), _p(mbump))
            assert rc == 0, rc

    def gpu_layout(self):
        """(root, nodes, instances, tris) copies of the reference adapters' output."""
        from imbatracer_b200.native import INST_DTYPE, NODE2_DTYPE
        root = C.c_int(0)
        pn, pi, pt = C.c_void_p(), C.c_void_p(), C.c_void_p()
        sizes = np.zeros(3, np.int64)
        self.lib.ref_scene_gpu_layout(self.handle, C.byref(root), C.byref(pn), C.byref(pi), C.byref(pt), _p(sizes))

        def grab(ptr, n, dtype):
            buf = (C.c_char * (int(n) * dtype.itemsize)).from_address(ptr)
            return np.frombuffer(bytes(buf), dtype=dtype).copy()

        # The reference over-allocates the node array (scene.cpp:14): keep the reachable range.
        nodes = grab(pn.value, sizes[0], NODE2_DTYPE)
        insts = grab(pi.value, sizes[1], INST_DTYPE)
        tris = grab(pt.value, sizes[2], np.dtype((np.float32, 4)))
        return root.value, nodes, insts, tris

    @classmethod
    def from_file(cls, path, width=512, height=512, fov=60.0):
        """A scene built by the reference's own frontend (build_scene.cpp) from a .scene file."""
        from types import SimpleNamespace

        from imbatracer_b200 import scenegen as G
        self = cls.__new__(cls)
        self.lib = load()
        cam9 = np.zeros(9, np.float32)
        self.handle = self.lib.ref_scene_load(os.fsencode(path), _p(cam9))
        if not self.handle:
            raise RuntimeError(f"the reference could not load {path}")
        cam = G.Camera(tuple(map(float, cam9[0:3])), tuple(map(float, cam9[3:6])), tuple(map(float, cam9[6:9])),
                       fov, width, height)
        self.desc = SimpleNamespace(camera=cam)
        return self

    def export(self) -> dict:
        """The arrays of the reference's scene (ref_scene_io.cpp): meshes, instances,
        materials, lights, textures, masks."""
        cnt = np.zeros(10, np.int64)
        lib = self.lib
        lib.ref_scene_counts(self.handle, _p(cnt))
        n_mesh, nv, nt, ni, nm, nl, ntex, texels, nmask, nbuf = (int(c) for c in cnt)
        out = {"mesh_counts": np.zeros((n_mesh, 2), np.int32), "vertices": np.zeros((nv, 3), np.float32),
               "normals": np.zeros((nv, 3), np.float32), "texcoords": np.zeros((nv, 2), np.float32),
               "indices": np.zeros((nt, 4), np.int32), "geom_normals": np.zeros((nt, 3), np.float32),
               "inst_mesh": np.zeros(ni, np.int32), "inst_mats": np.zeros((ni, 4, 4), np.float32),
               "mat_kind": np.zeros(nm, np.int32), "mat_params": np.zeros((nm, 16), np.float32),
               "light_kind": np.zeros(nl, np.int32), "light_params": np.zeros((nl, 12), np.float32),
               "tex_dims": np.zeros((max(ntex, 1), 2), np.int32), "texels": np.zeros((max(texels, 1), 4), np.float32),
               "masks": np.zeros((max(nmask, 1), 3), np.int32), "mask_buffer": np.zeros(max(nbuf, 1), np.uint8)}
        lib.ref_scene_meshes(self.handle, _p(out["mesh_counts"]), _p(out["vertices"]), _p(out["normals"]),
                             _p(out["texcoords"]), _p(out["indices"]), _p(out["geom_normals"]))
        lib.ref_scene_instances(self.handle, _p(out["inst_mesh"]), _p(out["inst_mats"]))
        assert lib.ref_scene_materials(self.handle, _p(out["mat_kind"]), _p(out["mat_params"])) == 0
        assert lib.ref_scene_lights(self.handle, _p(out["light_kind"]), _p(out["light_params"])) == 0
        lib.ref_scene_textures(self.handle, _p(out["tex_dims"]), _p(out["texels"]))
        lib.ref_scene_masks(self.handle, _p(out["masks"]), _p(out["mask_buffer"]))
        dims, inten = np.zeros(2, np.int32), np.zeros(1, np.float32)
        if lib.ref_scene_env(self.handle, _p(dims), None, _p(inten)) == 0:
            tex = np.zeros((int(dims[1]) * int(dims[0]), 4), np.float32)
            lib.ref_scene_env(self.handle, _p(dims), _p(tex), _p(inten))
            out["env_dims"], out["env_texels"], out["env_intensity"] = dims, tex, float(inten[0])
        out["tex_dims"] = out["tex_dims"][:ntex]
        out["texels"] = out["texels"][:texels]
        out["masks"] = out["masks"][:nmask]
        out["mask_buffer"] = out["mask_buffer"][:nbuf]
        return out

    def cpu_layout(self):
        """(root, nodes, instances, tris) of the reference CPU adapters (cpu_buffers=True)."""
        from imbatracer_b200.native import INST_DTYPE, NODE4_DTYPE
        root = C.c_int(0)
        pn, pi, pt = C.c_void_p(), C.c_void_p(), C.c_void_p()
        sizes = np.zeros(3, np.int64)
        assert self.lib.ref_scene_cpu_layout(self.handle, C.byref(root), C.byref(pn), C.byref(pi), C.byref(pt),
                                           _p(sizes)) == 0

        def grab(ptr, n, dtype):
            buf = (C.c_char * (int(n) * dtype.itemsize)).from_address(ptr)
            return np.frombuffer(bytes(buf), dtype=dtype).copy()

        return (root.value, grab(pn.value, sizes[0], NODE4_DTYPE), grab(pi.value, sizes[1], INST_DTYPE),
                grab(pt.value, sizes[2], np.dtype((np.float32, 4))))

    def render_pt(self, w, h, spp, max_path_len, seed_base, cam=None):
        cam = cam or self.desc.camera
        img = np.zeros((h, w, 3), np.float32)
        p3, d3, u3 = (np.ascontiguousarray(np.asarray(v, np.float32)) for v in (cam.pos, cam.dir, cam.up))
        rc = self.lib.ref_render_pt(self.handle, w, h, _p(p3), _p(d3), _p(u3), cam.fov, spp, max_path_len, seed_base,
                                  _p(img))
        assert rc == 0
        return img

    def render_pt_rr(self, w, h, spp, max_path_len, rr_start, seed_base, cam=None):
        """render_pt with the reference PathTracer's Russian roulette deferred to bounce
        rr_start (ref_pt_rr.cpp): no roulette draw and no kill before it; rr_start 0 is the
        reference itself."""
        cam = cam or self.desc.camera
        img = np.zeros((h, w, 3), np.float32)
        p3, d3, u3 = (np.ascontiguousarray(np.asarray(v, np.float32)) for v in (cam.pos, cam.dir, cam.up))
        rc = self.lib.ref_render_pt_rr(self.handle, w, h, _p(p3), _p(d3), _p(u3), cam.fov, spp, max_path_len, rr_start,
                                     seed_base, _p(img))
        assert rc == 0
        return img

    def render_pt_threads(self, w, h, spp, max_path_len, seed_base, threads, tile=32, cam=None):
        """The reference PT with `threads` tile threads; returns (image, closest rays, shadow
        rays) with the ray counts of the reference's own TileScheduler statistics."""
        cam = cam or self.desc.camera
        img = np.zeros((h, w, 3), np.float32)
        counts = np.zeros(2, np.int64)
        p3, d3, u3 = (np.ascontiguousarray(np.asarray(v, np.float32)) for v in (cam.pos, cam.dir, cam.up))
        self.lib.imbart_ref_set_threads(1, 1)
        rc = self.lib.ref_render_pt_threads(self.handle, w, h, _p(p3), _p(d3), _p(u3), cam.fov, spp, max_path_len,
                                          seed_base, tile, threads, _p(img), _p(counts))
        assert rc == 0
        return img, int(counts[0]), int(counts[1])

    def close(self):
        if self.handle:
            self.lib.ref_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


VCM_ALGOS = {"vcm": 0, "bpt": 1, "ppm": 2, "lt": 3, "pt": 4}


class RefVcm:
    """The reference's VCMIntegrator<algo> (vcm.cpp) on a RefScene, driven pass by pass.

    One camera tile covers the image (sample indices global); each light's paths form one
    light tile when tile_size^2 is at least the paths per light. Light vertices are 28 floats:
    pos, mat | out_dir, path_length | normal, dVC | geom_normal, dVCM | u_tangent, dVM |
    v_tangent, uv.x | throughput, uv.y (mat and path_length as int32 bits)."""

    def __init__(self, scene: RefScene, algo: str, w: int, h: int, spp: int = 1, max_path_len: int = 8,
                 light_path_count: int = 1024, num_connections: int = 1, num_knn: int = 10,
                 radius_factor: float = 2.0, tile_size: int | None = None, cam=None, preprocess_seed: int = 77):
        cam = cam or scene.desc.camera
        self.scene, self.w, self.h = scene, w, h
        self.light_path_count = light_path_count
        tile = tile_size or max(w, h, int(np.ceil(np.sqrt(light_path_count))) + 1)
        self.tile_size = tile
        p3, d3, u3 = (np.ascontiguousarray(np.asarray(v, np.float32)) for v in (cam.pos, cam.dir, cam.up))
        self.handle = load().ref_vcm_create(scene.handle, VCM_ALGOS[algo], w, h, _p(p3), _p(d3), _p(u3), cam.fov,
                                            spp, max_path_len, light_path_count, num_connections, num_knn,
                                            radius_factor, tile, preprocess_seed)
        assert self.handle
        info = np.zeros(3, np.float32)
        load().ref_vcm_info(self.handle, _p(info))
        self.pixel_size, self.base_radius, self.cache_capacity = float(info[0]), float(info[1]), int(info[2])

    def begin_iteration(self, iteration: int):
        eta = np.zeros(2, np.float32)
        r = load().ref_vcm_begin_iteration(self.handle, iteration, _p(eta))
        return float(r), float(eta[0]), float(eta[1])

    def light_pass(self, seed: int, step: int = 0) -> np.ndarray:
        img = np.zeros((self.h, self.w, 3), np.float32)
        load().ref_vcm_light_pass(self.handle, seed & (2 ** 64 - 1), step & (2 ** 64 - 1), _p(img))
        return img

    def light_vertices(self) -> np.ndarray:
        cap = max(self.cache_capacity, 1)
        out = np.zeros((cap, 28), np.float32)
        n = load().ref_vcm_light_vertices(self.handle, _p(out), cap)
        return out[:n].copy()

    def camera_pass(self, seed: int) -> np.ndarray:
        img = np.zeros((self.h, self.w, 3), np.float32)
        load().ref_vcm_camera_pass(self.handle, seed & (2 ** 64 - 1), _p(img))
        return img

    def time_grid(self, reps: int = 3, threads: int = 1) -> dict:
        """The reference's photon grid over the current cache: seconds per rebuild, and the
        seconds of one k-nearest query at every cached vertex on `threads` threads."""
        out = np.zeros(3, np.float64)
        load().ref_vcm_time_grid(self.handle, reps, threads, _p(out))
        return {"build_s": float(out[0]), "query_s": float(out[1]), "queries": int(out[2])}

    def close(self):
        if self.handle:
            load().ref_vcm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
