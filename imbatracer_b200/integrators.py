"""Host-side mirror of the reference's integrator interface for the wavefront path tracer.

    pt = PathTracer(desc, max_path_len=5)          # PathTracer(scene, cam, scheduler, max_path_len), pt.h:20-25
    image = pt.render(spp=4, seed_base=7)          # Integrator::render(AtomicImage&), pt.cpp:162-178

The scene is prepared once on the GPU (8-wide BVH + shading data); render() runs one frame
entirely on the device (sample generation, traversal, shading, shadow rays) and returns
the accumulated radiance as a (height, width, 3) float32 CUDA tensor, like the reference's
AtomicImage after one frame. There is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from . import scene as S
from . import scenegen as G


class ShadingData:
    """Global shading arrays of a SceneDesc (vertices, normals, texcoords, triangles with
    global vertex indices and materials, instances, materials, lights, environment)."""

    def __init__(self, desc: G.SceneDesc):
        voff, verts, nrms, tcs, tris, gns = 0, [], [], [], [], []
        for m in desc.meshes:
            verts.append(m.vertices)
            nrms.append(m.normals)
            tcs.append(m.texcoords)
            t = m.indices.copy()
            t[:, :3] += voff
            tris.append(t)
            gns.append(m.geom_normals)
            voff += len(m.vertices)
        self.vertices = np.ascontiguousarray(np.concatenate(verts), np.float32)
        self.normals = np.ascontiguousarray(np.concatenate(nrms), np.float32)
        self.texcoords = np.ascontiguousarray(np.concatenate(tcs), np.float32)
        self.tris = np.ascontiguousarray(np.concatenate(tris), np.int32)
        self.geom_normals = np.ascontiguousarray(np.concatenate(gns), np.float32)
        self.inst_inv = np.ascontiguousarray(np.stack([i.inv_mat.reshape(-1) for i in desc.instances]), np.float32)
        self.mat_kind = np.array([m.kind for m in desc.materials], np.int32)
        prm = np.zeros((len(desc.materials), 16), np.float32)
        for i, m in enumerate(desc.materials):
            prm[i, 0:3] = m.color
            prm[i, 3:6] = m.specular
            prm[i, 6] = m.exponent
            prm[i, 7] = m.eta
            prm[i, 8] = m.kappa
            prm[i, 9:12] = m.emission
            prm[i, 12] = getattr(m, "texture", -1)
            prm[i, 13] = getattr(m, "bump", -1)
        self.mat_params = prm
        n_tri, delta = len(desc.lights), list(getattr(desc, "delta_lights", []))
        rows = [(0, np.concatenate([p0, p1, p2, e]).astype(np.float32)) for p0, p1, p2, e in desc.lights]
        drows = [(k, np.asarray(prm12, np.float32)) for k, prm12 in delta]
        # Light order = the reference's light list: delta lights first for scenes read from
        # files (parse order), after the triangle lights otherwise.
        rows = drows + rows if getattr(desc, "delta_first", False) else rows + drows
        lights = np.zeros((max(len(rows), 1), 12), np.float32)
        for i, (_, r) in enumerate(rows):
            lights[i] = r
        self.lights = lights
        self.n_lights = len(rows)
        self.light_kinds = np.array([k for k, _ in rows] or [0], np.int32)
        tex = list(getattr(desc, "textures", []))
        self.n_textures = len(tex)
        self.tex_dims = np.array([[t.shape[1], t.shape[0]] for t in tex] or [[0, 0]], np.int32).reshape(-1)
        self.tex_pixels = (np.ascontiguousarray(np.concatenate([np.asarray(t, np.float32).reshape(-1) for t in tex]))
                           if tex else np.zeros(4, np.float32))
        self.env = None if desc.env_intensity is None else np.array(desc.env_intensity, np.float32)
        self.env_map = int(getattr(desc, "env_map", -1))
        self.env_map_intensity = float(getattr(desc, "env_map_intensity", 1.0))
        if self.env_map >= 0 and self.env is None:
            self.env = np.zeros(3, np.float32)     # the environment light exists; its image is set after
        self.bsphere = bounding_sphere(desc)


def bounding_sphere(desc) -> np.ndarray:
    """Scene::compute_bounding_sphere (scene.cpp:189-200): the union of the instances' mesh
    boxes transformed by transform(float3x4, BBox) (float3x4.h:52-56: centre and half extent
    through the matrix and its absolute value); radius = half the diagonal. Evaluated in
    single precision in the reference's operation order, so the sphere is the reference's.
    Returns centre xyz, radius, 1 / radius^2."""
    f = np.float32
    lo = [f(np.inf)] * 3
    hi = [f(-np.inf)] * 3
    half = f(0.5)
    for inst in desc.instances:
        mlo, mhi = desc.meshes[inst.mesh_id].bounding_box()
        m = inst.mat.astype(np.float32)
        c3 = [f(f(mhi[k] + mlo[k]) * half) for k in range(3)]
        e3 = [f(f(mhi[k] - mlo[k]) * half) for k in range(3)]
        for r in range(3):
            c = f(f(f(f(m[r, 0] * c3[0]) + f(m[r, 1] * c3[1])) + f(m[r, 2] * c3[2])) + f(m[r, 3] * f(1.0)))
            a = [f(abs(m[r, k])) for k in range(4)]
            e = f(f(f(f(a[0] * e3[0]) + f(a[1] * e3[1])) + f(a[2] * e3[2])) + f(a[3] * f(0.0)))
            lo[r] = min(lo[r], f(c - e))
            hi[r] = max(hi[r], f(c + e))
    d = [f(hi[k] - lo[k]) for k in range(3)]
    r = f(f(np.sqrt(f(f(f(d[0] * d[0]) + f(d[1] * d[1])) + f(d[2] * d[2])))) * half)
    c = [f(f(hi[k] + lo[k]) * half) for k in range(3)]
    return np.array([c[0], c[1], c[2], r, f(f(1.0) / f(r * r))], np.float32)


class GpuScene:
    """A SceneDesc resident on one GPU: traversal scene + shading data."""

    def __init__(self, desc: G.SceneDesc, device: int = 0, td: S.TraversalData | None = None,
                 gpu_build: bool = False):
        """gpu_build: build the BVHs on the GPU (imbart_scene_build_gpu; unmasked scenes)
        instead of the host SBVH builder and layout conversion."""
        self.desc = desc
        self.device = device
        if gpu_build:
            if getattr(desc, "masks", None) is not None and (desc.masks["width"] * desc.masks["height"] > 1).any():
                raise N.ImbartError("GpuScene: the GPU builder does not take opacity masks")
            self.td = None
            self.trace_scene = S.DeviceScene.build_gpu(desc.meshes, desc.instances, device)
        else:
            self.td = td if td is not None else S.build_traversal_data(
                desc.meshes, desc.instances, masks=getattr(desc, "masks", None),
                mask_buffer=getattr(desc, "mask_buffer", None), accel_files=getattr(desc, "accel_files", None))
            self.trace_scene = S.DeviceScene(self.td, device)
        sd = ShadingData(desc)
        self.sd = sd
        lib = N.load()
        h = lib.imbart_shading_create_ex(device, N.ptr(sd.vertices), len(sd.vertices), N.ptr(sd.normals),
                                         N.ptr(sd.texcoords), N.ptr(sd.tris), N.ptr(sd.geom_normals), len(sd.tris),
                                         N.ptr(sd.inst_inv), len(sd.inst_inv), N.ptr(sd.mat_kind),
                                         N.ptr(sd.mat_params), len(sd.mat_kind), N.ptr(sd.light_kinds),
                                         N.ptr(sd.lights), sd.n_lights, N.ptr(sd.env), N.ptr(sd.bsphere),
                                         N.ptr(sd.tex_dims), N.ptr(sd.tex_pixels), sd.n_textures)
        if not h:
            raise N.ImbartError("imbart_shading_create: " + N.last_error()[1])
        self.shading = h
        if sd.env_map >= 0:
            N.check(lib.imbart_shading_set_env_map(h, sd.env_map, sd.env_map_intensity), "imbart_shading_set_env_map")

    def autotune_node_width(self, ray_sets, stream=None, widths=(8, 4)) -> dict:
        """Chooses the node width with the autotuner: the scene is prepared at each width from
        the same reference-layout arrays, each query class in `ray_sets` ((rays, hits, flags)
        device tensors) is tuned on it (imbart_trace_autotune, from the same starting
        configuration), and the width whose tuned kernels trace all classes fastest is kept
        with its configuration. Call before creating integrators on this scene (they hold
        its traversal handle). Host-built scenes only."""
        if self.td is None:
            raise N.ImbartError("autotune_node_width: the scene was built on the GPU (8-wide only)")
        start = S.trace_config_snapshot()
        results, best = {}, None
        for w in widths:
            scene = self.trace_scene if self.trace_scene.node_width == w else S.DeviceScene(self.td, self.device,
                                                                                            node_width=w)
            S.trace_config_restore(start)
            classes = {}
            try:
                for rays, hits, flags in ray_sets:
                    classes[flags] = scene.autotune(rays, hits, flags, stream=stream)
            except Exception:
                S.trace_config_restore(start)
                for sc in (scene, best[1] if best else None):
                    if sc is not None and sc is not self.trace_scene:
                        sc.close()
                raise
            total = sum(c["ms"] for c in classes.values())
            results[w] = {"ms": total, "classes": classes, "config": S.trace_config_snapshot()}
            if best is None or total < results[best[0]]["ms"]:
                if best is not None and best[1] is not self.trace_scene:
                    best[1].close()
                best = (w, scene)
            elif scene is not self.trace_scene:
                scene.close()
        w, scene = best
        if scene is not self.trace_scene:
            self.trace_scene.close()
            self.trace_scene = scene
        S.trace_config_restore(results[w]["config"])
        return {"node_width": w, "ms": {k: round(v["ms"], 4) for k, v in results.items()},
                "classes": results[w]["classes"]}

    def close(self):
        if getattr(self, "shading", None):
            N.load().imbart_shading_destroy(self.shading)
            self.shading = None
        self.trace_scene.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def camera_matrix(cam: G.Camera, width: int | None = None, height: int | None = None) -> np.ndarray:
    """raster_to_world of PerspectiveCamera(w, h, fov).move(pos, dir, up) (camera.h:27-56)."""
    w = float(width or cam.width)
    h = float(height or cam.height)
    r2w = np.zeros(16, np.float32)
    f = lambda v: np.ascontiguousarray(np.asarray(v, np.float32))
    p, d, u = f(cam.pos), f(cam.dir), f(cam.up)
    N.check(N.load().imbart_camera_setup(N.ptr(p), N.ptr(d), N.ptr(u), float(cam.fov), w, h, 1.0, N.ptr(r2w), None,
                                         None), "imbart_camera_setup")
    return r2w


class PathTracer:
    """Wavefront path tracer (pt.cpp) on the GPU."""

    def __init__(self, scene: GpuScene, max_path_len: int = 10, rr_start: int = 0, max_paths_in_flight: int = 0,
                 graphs: int | None = None):
        """graphs: each sample range's bounce loop driven from the host (0), as a CUDA graph
        (1), as a CUDA graph with the shadow-ray work on a branch of its own (2), or as
        IMBART_PT_GRAPH says (None; default 2)."""
        self.scene = scene
        self.max_path_len = max_path_len
        self.rr_start = rr_start
        self.max_paths = max_paths_in_flight
        lib = N.load()
        self.ctx = lib.imbart_pt_create(scene.device)
        if not self.ctx:
            raise N.ImbartError("imbart_pt_create: " + N.last_error()[1])
        N.check(lib.imbart_pt_set_graphs(self.ctx, -1 if graphs is None else int(graphs)),
                "imbart_pt_set_graphs")
        self.last_stats = np.zeros(3, np.int64)

    def render(self, spp: int, seed_base: int, width: int | None = None, height: int | None = None, image=None,
               stream=None, cam: G.Camera | None = None, stats: bool = True, sample_range=None):
        """Adds one frame to `image` (a new zeroed image when None) on `stream`. With stats,
        last_stats holds the frame's closest-hit rays, shadow rays and wavefronts (one
        synchronization at the end); without, a graph-driven frame returns unsynchronized.
        sample_range (first, count): only those of the frame's width * height * spp samples
        (imbart_pt_render_range), seeded as in the whole frame."""
        import torch
        cam = cam or self.scene.desc.camera
        w = width or cam.width
        h = height or cam.height
        r2w = camera_matrix(cam, w, h)
        pos = np.ascontiguousarray(np.asarray(cam.pos, np.float32))
        dev = torch.device("cuda", self.scene.device)
        if image is None:
            image = torch.zeros((h, w, 3), dtype=torch.float32, device=dev)
        st = None if stream is None else stream.cuda_stream
        out = np.zeros(3, np.int64)
        if sample_range is None:
            N.check(N.load().imbart_pt_render(self.ctx, self.scene.trace_scene.handle, self.scene.shading, N.ptr(r2w),
                                              N.ptr(pos), w, h, spp, self.max_path_len, self.rr_start,
                                              seed_base & (2 ** 64 - 1), N.ptr(image), self.max_paths,
                                              N.ptr(out) if stats else None, st),
                    "imbart_pt_render")
        else:
            first, count = (int(v) for v in sample_range)
            N.check(N.load().imbart_pt_render_range(self.ctx, self.scene.trace_scene.handle, self.scene.shading,
                                                    N.ptr(r2w), N.ptr(pos), w, h, spp, self.max_path_len,
                                                    self.rr_start, seed_base & (2 ** 64 - 1), N.ptr(image),
                                                    self.max_paths, first, count, N.ptr(out) if stats else None,
                                                    st),
                    "imbart_pt_render_range")
        if stats:
            self.last_stats = out
        return image

    def autotune_wavefront(self, spp: int, seed_base: int = 0, width: int | None = None, height: int | None = None,
                           sizes=(4 << 20, 8 << 20, 16 << 20, 32 << 20), repeats: int = 2, stream=None):
        """Picks the wavefront size (paths in flight) for frames of this shape: one untimed
        frame per size (it grows the queues and builds the graph), then `repeats` frames timed
        with CUDA events on the stream; keeps the fastest in max_paths_in_flight. Returns
        {size: ms per frame}."""
        import torch
        cam = self.scene.desc.camera
        w, h = width or cam.width, height or cam.height
        dev = torch.device("cuda", self.scene.device)
        st = stream or torch.cuda.current_stream(dev)
        image = torch.zeros((h, w, 3), dtype=torch.float32, device=dev)
        total = w * h * spp
        times = {}
        for size in sizes:
            size = int(min(size, total))
            if size in times:
                continue
            self.max_paths = size
            self.render(spp, seed_base, w, h, image=image, stream=st)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for k in range(repeats):
                self.render(spp, seed_base + 1 + k, w, h, image=image, stream=st)
            e1.record(st)
            e1.synchronize()
            times[size] = e0.elapsed_time(e1) / repeats
        self.max_paths = min(times, key=times.get)
        return times

    def close(self):
        if getattr(self, "ctx", None):
            N.load().imbart_pt_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_camera(cam: G.Camera, width: int | None = None, height: int | None = None) -> N.Camera:
    """PerspectiveCamera(width, height, fov).move(pos, dir, up) (camera.h:20-56)."""
    c = N.Camera()
    f = lambda v: np.ascontiguousarray(np.asarray(v, np.float32))
    p, d, u = f(cam.pos), f(cam.dir), f(cam.up)
    N.check(N.load().imbart_camera_make(N.ptr(p), N.ptr(d), N.ptr(u), float(cam.fov), int(width or cam.width),
                                        int(height or cam.height), C.byref(c)), "imbart_camera_make")
    return c


def estimate_pixel_size(scene: GpuScene, cam: N.Camera) -> float:
    """Integrator::estimate_pixel_size (integrator.cpp:14-70) on the GPU."""
    out = np.zeros(1, np.float32)
    N.check(N.load().imbart_estimate_pixel_size(scene.trace_scene.handle, C.byref(cam), N.ptr(out), None),
            "imbart_estimate_pixel_size")
    return float(out[0])


class VcmIntegrator:
    """VCMIntegrator<algo> (vcm.h:54-150) on the GPU: algorithm "vcm", "bpt", "ppm", "lt" or
    "pt"; settings as the reference's UserSettings (cmd_line.h:40-58). render(iteration) =
    light pass + camera pass (vcm.cpp:25-55); the photon radius shrinks with the iteration
    (base_radius * i^-radius_exponent; 0 = the reference's 1/8) and the photon grid has cells
    of grid_cell_factor radii (0 = the reference's 2) and grid_table_size buckets (0 = twice
    the photons).
    Images are (height, width, 3) float32 CUDA tensors, accumulated like the reference's
    AtomicImage."""

    def __init__(self, scene: GpuScene, algorithm: str = "vcm", width: int | None = None, height: int | None = None,
                 spp: int = 1, max_path_len: int = 10, light_path_count: int | None = None,
                 num_connections: int = 1, num_knn: int = 10, radius_factor: float = 2.0,
                 base_radius: float | None = None, light_tile_size: int = 0, cam: G.Camera | None = None,
                 max_paths_in_flight: int = 0, radius_exponent: float = 0.0, grid_cell_factor: float = 0.0,
                 grid_table_size: int = 0):
        self.scene = scene
        cam = cam or scene.desc.camera
        self.width = width or cam.width
        self.height = height or cam.height
        self.camera = make_camera(cam, self.width, self.height)
        st = self.settings = N.VcmSettings()
        st.algorithm = N.VCM_ALGORITHMS[algorithm]
        st.spp = spp
        st.max_path_len = max_path_len
        st.light_path_count = light_path_count or (self.width * self.height // 2)
        st.num_connections = num_connections
        st.num_knn = num_knn
        st.light_tile_size = light_tile_size
        self.pixel_size = estimate_pixel_size(scene, self.camera)
        st.base_radius = base_radius if base_radius is not None else self.pixel_size * radius_factor
        # Photon-grid schedule; zeros keep the reference's (radius ~ i^-1/8, cell 2r, 2n buckets).
        st.radius_exponent = radius_exponent
        st.grid_cell_factor = grid_cell_factor
        st.grid_table_size = grid_table_size
        self.max_paths = max_paths_in_flight
        self.ctx = N.load().imbart_vcm_create(scene.device)
        if not self.ctx:
            raise N.ImbartError("imbart_vcm_create: " + N.last_error()[1])
        self.last_stats = np.zeros(6, np.int64)

    def _image(self, image):
        import torch
        if image is None:
            image = torch.zeros((self.height, self.width, 3), dtype=torch.float32,
                                device=torch.device("cuda", self.scene.device))
        return image

    def begin_iteration(self, iteration: int):
        """Returns (photon radius, eta_vc, eta_vm) of the iteration."""
        out = np.zeros(3, np.float32)
        N.check(N.load().imbart_vcm_begin_iteration(self.ctx, C.byref(self.settings), iteration, N.ptr(out)),
                "imbart_vcm_begin_iteration")
        return float(out[0]), float(out[1]), float(out[2])

    def light_pass(self, light_seed: int, light_seed_step: int = 0, image=None):
        image = self._image(image)
        self.settings.light_seed = light_seed & (2 ** 64 - 1)
        self.settings.light_seed_step = light_seed_step & (2 ** 64 - 1)
        stats = np.zeros(3, np.int64)
        N.check(N.load().imbart_vcm_light_pass(self.ctx, self.scene.trace_scene.handle, self.scene.shading,
                                               C.byref(self.camera), C.byref(self.settings), N.ptr(image),
                                               N.ptr(stats), None), "imbart_vcm_light_pass")
        self.last_stats[:3] = stats
        return image

    def camera_pass(self, camera_seed: int, image=None):
        image = self._image(image)
        self.settings.camera_seed = camera_seed & (2 ** 64 - 1)
        stats = np.zeros(3, np.int64)
        N.check(N.load().imbart_vcm_camera_pass(self.ctx, self.scene.trace_scene.handle, self.scene.shading,
                                                C.byref(self.camera), C.byref(self.settings), N.ptr(image),
                                                self.max_paths, N.ptr(stats), None), "imbart_vcm_camera_pass")
        self.last_stats[3:] = stats
        return image

    def render(self, iteration: int, light_seed: int, camera_seed: int, light_seed_step: int = 0, image=None):
        image = self._image(image)
        self.settings.light_seed = light_seed & (2 ** 64 - 1)
        self.settings.light_seed_step = light_seed_step & (2 ** 64 - 1)
        self.settings.camera_seed = camera_seed & (2 ** 64 - 1)
        stats = np.zeros(3, np.int64)
        N.check(N.load().imbart_vcm_render(self.ctx, self.scene.trace_scene.handle, self.scene.shading,
                                           C.byref(self.camera), C.byref(self.settings), iteration, N.ptr(image),
                                           self.max_paths, N.ptr(stats), None), "imbart_vcm_render")
        self.last_stats[:3] = stats
        return image

    def light_vertices(self) -> np.ndarray:
        """The light-vertex cache as a (count, 28) float32 host array (layout: include/imbart.h)."""
        lib = N.load()
        n = lib.imbart_vcm_copy_light_vertices(self.ctx, None, 0)
        if n < 0:
            raise N.ImbartError("imbart_vcm_copy_light_vertices: " + N.last_error()[1])
        out = np.zeros((n, 28), np.float32)
        if n > 0 and lib.imbart_vcm_copy_light_vertices(self.ctx, N.ptr(out), n) != n:
            raise N.ImbartError("imbart_vcm_copy_light_vertices: " + N.last_error()[1])
        return out

    def load_light_vertices(self, vertices) -> None:
        """Replaces the cache (e.g. with the reference's, or the vertices of several GPUs) and
        rebuilds the photon grid. vertices: (count, 28) float32 host array or CUDA tensor."""
        if isinstance(vertices, np.ndarray):
            vertices = np.ascontiguousarray(vertices, np.float32).reshape(-1, 28)
        else:
            vertices = vertices.contiguous().view(-1, 28)
        N.check(N.load().imbart_vcm_load_light_vertices(self.ctx, C.byref(self.settings), N.ptr(vertices),
                                                        int(vertices.shape[0]), None), "imbart_vcm_load_light_vertices")

    def light_pass_range(self, first_path: int, n_paths: int, light_seed: int, light_seed_step: int = 0,
                         image=None):
        """The light pass over paths [first_path, first_path + n_paths) of the iteration; returns
        (image, vertices added per wavefront)."""
        image = self._image(image)
        self.settings.light_seed = light_seed & (2 ** 64 - 1)
        self.settings.light_seed_step = light_seed_step & (2 ** 64 - 1)
        stats = np.zeros(3, np.int64)
        waves = np.zeros(self.settings.max_path_len + 1, np.int32)
        N.check(N.load().imbart_vcm_light_pass_range(self.ctx, self.scene.trace_scene.handle, self.scene.shading,
                                                     C.byref(self.camera), C.byref(self.settings), first_path,
                                                     n_paths, N.ptr(image), N.ptr(waves), len(waves), N.ptr(stats),
                                                     None), "imbart_vcm_light_pass_range")
        self.last_stats[:3] = stats
        return image, waves

    def camera_pass_range(self, first_sample: int, n_samples: int, camera_seed: int, image=None):
        image = self._image(image)
        self.settings.camera_seed = camera_seed & (2 ** 64 - 1)
        stats = np.zeros(3, np.int64)
        N.check(N.load().imbart_vcm_camera_pass_range(self.ctx, self.scene.trace_scene.handle, self.scene.shading,
                                                      C.byref(self.camera), C.byref(self.settings), first_sample,
                                                      n_samples, N.ptr(image), self.max_paths, N.ptr(stats), None),
                "imbart_vcm_camera_pass_range")
        self.last_stats[3:] = stats
        return image

    def light_vertices_device(self):
        """The cache as a (count, 28) float32 CUDA tensor (a copy)."""
        import torch
        ptr, n = C.c_void_p(), C.c_int(0)
        N.check(N.load().imbart_vcm_light_vertices(self.ctx, C.byref(ptr), C.byref(n)), "imbart_vcm_light_vertices")
        out = torch.empty((n.value, 28), dtype=torch.float32, device=torch.device("cuda", self.scene.device))
        if n.value > 0:
            class _View:
                __cuda_array_interface__ = {"shape": (n.value, 28), "typestr": "<f4", "data": (ptr.value, False),
                                            "version": 3}
            out.copy_(torch.as_tensor(_View(), device=out.device))
        return out

    def close(self):
        if getattr(self, "ctx", None):
            N.load().imbart_vcm_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
