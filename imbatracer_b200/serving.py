"""Request server over libimbart's imbart_server_* entry points (include/imbart.h).

    srv = Server(mode="batched", hbm_budget=8 << 30)
    sid = srv.add_scene(desc)                              # SceneDesc from scenegen
    t, img = srv.submit_render(sid, desc.camera, 256, 256, spp=4, max_path_len=5, seed_base=1)
    res = srv.wait(t)                                      # img (host numpy) is now filled

"batched" merges the wavefronts of all admitted requests over all resident scenes (one pool
of `hbm_budget` bytes with LRU eviction); "plain" serves the same requests one at a time
through imbart_pt_render / imbart_trace. Both run on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import native as N
from . import scene as S
from . import scenegen as G
from .integrators import ShadingData, camera_matrix, make_camera

MODES = {"batched": N.SERVE_BATCHED, "plain": N.SERVE_PLAIN}


class Server:
    def __init__(self, device: int = 0, mode: str = "batched", hbm_budget: int = 4 << 30, max_paths: int = 4 << 20):
        self.lib = N.load()
        self.mode = mode
        self.h = self.lib.imbart_server_create(device, MODES[mode], int(hbm_budget), int(max_paths))
        if not self.h:
            raise N.ImbartError("imbart_server_create: " + N.last_error()[1])
        self._keep = {}            # ticket -> buffers the server still reads or writes
        self._scenes = []          # host arrays of registered scenes (the server copies them; kept for reuse)
        self._lock = threading.Lock()

    def add_scene(self, desc: G.SceneDesc, td: S.TraversalData | None = None, gpu_build: bool = False) -> int:
        """Registers a scene: its traversal arrays from `td` (built on the host when None) or,
        with gpu_build, built on the server's GPU (imbart_server_add_scene_gpu_build; the
        build's wall time is then in last_build_ms)."""
        masks = getattr(desc, "masks", None)
        if masks is not None and (np.asarray(masks["width"]) * np.asarray(masks["height"]) > 1).any():
            raise N.ImbartError("imbart_server_add_scene: opacity masks are not supported by the server")
        if not gpu_build:
            td = td if td is not None else S.build_traversal_data(desc.meshes, desc.instances,
                                                                  accel_files=getattr(desc, "accel_files", None))
        sd = ShadingData(desc)
        src = N.SceneSource()
        if not gpu_build:
            src.root = td.root
            src.nodes, src.n_nodes = N.ptr(td.nodes), len(td.nodes)
            src.instances, src.n_instances = N.ptr(td.instances), len(td.instances)
            src.tris, src.n_tri_vec4 = N.ptr(td.tris), len(td.tris)
        src.vertices, src.n_vertices = N.ptr(sd.vertices), len(sd.vertices)
        src.normals, src.texcoords = N.ptr(sd.normals), N.ptr(sd.texcoords)
        src.mesh_tris, src.geom_normals, src.n_mesh_tris = N.ptr(sd.tris), N.ptr(sd.geom_normals), len(sd.tris)
        src.inst_inv, src.n_inst_inv = N.ptr(sd.inst_inv), len(sd.inst_inv)
        src.mat_kind, src.mat_params, src.n_mats = N.ptr(sd.mat_kind), N.ptr(sd.mat_params), len(sd.mat_kind)
        src.tri_lights, src.n_tri_lights = N.ptr(sd.lights), sd.n_lights
        src.env_color, src.bsphere = N.ptr(sd.env), N.ptr(sd.bsphere)
        src.light_kinds = N.ptr(sd.light_kinds)
        src.tex_dims, src.tex_pixels, src.n_textures = N.ptr(sd.tex_dims), N.ptr(sd.tex_pixels), sd.n_textures
        src.env_map, src.env_intensity = sd.env_map + 1, sd.env_map_intensity
        self._scenes.append((td, sd))   # the arrays the source points to stay alive during the call
        if gpu_build:
            md, idesc, keep = S.build_descs(desc.meshes, desc.instances)
            ms = C.c_float(0.0)
            sid = self.lib.imbart_server_add_scene_gpu_build(self.h, C.byref(src), md, len(desc.meshes), idesc,
                                                             len(desc.instances), C.byref(ms))
            self.last_build_ms = ms.value
        else:
            sid = self.lib.imbart_server_add_scene(self.h, C.byref(src))
        if sid < 0:
            raise N.ImbartError("imbart_server_add_scene: " + N.last_error()[1])
        return sid

    def submit_render(self, scene: int, cam: G.Camera, width: int, height: int, spp: int, max_path_len: int,
                      seed_base: int, rr_start: int = 0, image: np.ndarray | None = None):
        """Returns (ticket, image): `image` (height, width, 3) float32 host array, filled when
        the request completes."""
        if image is None:
            image = np.zeros((height, width, 3), np.float32)
        assert image.dtype == np.float32 and image.flags.c_contiguous and image.size == width * height * 3
        q = N.RenderRequest()
        q.scene = scene
        q.raster_to_world[:] = [float(v) for v in camera_matrix(cam, width, height)]
        q.cam_pos[:] = [float(v) for v in cam.pos]
        q.width, q.height, q.spp, q.max_path_len, q.rr_start = width, height, spp, max_path_len, rr_start
        q.seed_base = seed_base & (2 ** 64 - 1)
        q.image_host = N.ptr(image)
        t = self.lib.imbart_server_submit_render(self.h, C.byref(q))
        if t < 0:
            raise N.ImbartError("imbart_server_submit_render: " + N.last_error()[1])
        with self._lock:
            self._keep[t] = image
        return t, image

    def submit_vcm(self, scene: int, cam: G.Camera, width: int, height: int, algorithm: str = "vcm",
                   iterations: int = 1, max_path_len: int = 8, light_path_count: int | None = None,
                   num_connections: int = 1, num_knn: int = 10, radius_factor: float = 2.0,
                   base_radius: float = 0.0, light_seed: int = 1, camera_seed: int = 2, seed_step: int = 1,
                   light_seed_step: int = 0x9E3779B9, light_tile_size: int = 0, image: np.ndarray | None = None):
        """A VCM-family frame ("vcm", "bpt", "ppm", "lt", "pt"): `iterations` iterations into
        one accumulated (height, width, 3) float32 host image. Returns (ticket, image).
        base_radius 0 takes radius_factor times the camera's estimated pixel size."""
        if image is None:
            image = np.zeros((height, width, 3), np.float32)
        assert image.dtype == np.float32 and image.flags.c_contiguous and image.size == width * height * 3
        q = N.VcmRequest()
        q.scene = scene
        q.camera = make_camera(cam, width, height)
        st = q.settings
        st.algorithm = N.VCM_ALGORITHMS[algorithm]
        st.spp = 1
        st.max_path_len = max_path_len
        st.light_path_count = light_path_count or (width * height // 2)
        st.num_connections = num_connections
        st.num_knn = num_knn
        st.light_tile_size = light_tile_size
        st.base_radius = base_radius
        st.light_seed = light_seed & (2 ** 64 - 1)
        st.light_seed_step = light_seed_step & (2 ** 64 - 1)
        st.camera_seed = camera_seed & (2 ** 64 - 1)
        q.radius_factor = radius_factor
        q.iterations = iterations
        q.seed_step = seed_step & (2 ** 64 - 1)
        q.image_host = N.ptr(image)
        t = self.lib.imbart_server_submit_vcm(self.h, C.byref(q))
        if t < 0:
            raise N.ImbartError("imbart_server_submit_vcm: " + N.last_error()[1])
        with self._lock:
            self._keep[t] = image
        return t, image

    def submit_rays(self, scene: int, rays, hits, flags: int = N.TRACE_CLOSEST) -> int:
        """rays / hits: numpy arrays (RAY_DTYPE / HIT_DTYPE, pageable or pinned) or CUDA
        tensors of the same byte layout."""
        n = len(rays)
        t = self.lib.imbart_server_submit_rays(self.h, scene, N.ptr(rays), N.ptr(hits), n, flags)
        if t < 0:
            raise N.ImbartError("imbart_server_submit_rays: " + N.last_error()[1])
        with self._lock:
            self._keep[t] = (rays, hits)
        return t

    def wait(self, ticket: int) -> dict:
        r = N.RequestResult()
        self.lib.imbart_server_wait(self.h, ticket, C.byref(r))
        with self._lock:
            self._keep.pop(ticket, None)
        return {"status": r.status, "kind": r.kind, "submit_ms": r.submit_ms, "start_ms": r.start_ms,
                "done_ms": r.done_ms}

    def drain(self) -> None:
        N.check(self.lib.imbart_server_drain(self.h), "imbart_server_drain")

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(self.lib.imbart_server_get_stats(self.h, C.byref(s)), "imbart_server_get_stats")
        return {k: getattr(s, k) for k, _ in N.ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.imbart_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
