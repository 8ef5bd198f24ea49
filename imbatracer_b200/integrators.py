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
        self.mat_params = prm
        lights = np.zeros((max(len(desc.lights), 1), 12), np.float32)
        for i, (p0, p1, p2, e) in enumerate(desc.lights):
            lights[i] = np.concatenate([p0, p1, p2, e])
        self.lights = lights
        self.n_lights = len(desc.lights)
        self.env = None if desc.env_intensity is None else np.array(desc.env_intensity, np.float32)
        self.bsphere = bounding_sphere(desc)


def bounding_sphere(desc) -> np.ndarray:
    """Scene::compute_bounding_sphere (scene.cpp:190-200): the box of the transformed mesh
    boxes; radius = half its diagonal."""
    lo = np.full(3, np.inf, np.float32)
    hi = np.full(3, -np.inf, np.float32)
    for inst in desc.instances:
        mlo, mhi = desc.meshes[inst.mesh_id].bounding_box()
        m = inst.mat[:3, :]
        c = m[:, :3] @ ((mhi + mlo) * np.float32(0.5)) + m[:, 3]
        e = np.abs(m[:, :3]) @ ((mhi - mlo) * np.float32(0.5))
        lo = np.minimum(lo, c - e)
        hi = np.maximum(hi, c + e)
    r = np.float32(np.linalg.norm(hi - lo) * 0.5)
    c = (hi + lo) * np.float32(0.5)
    return np.array([c[0], c[1], c[2], r, 1.0 / (r * r)], np.float32)


class GpuScene:
    """A SceneDesc resident on one GPU: traversal scene + shading data."""

    def __init__(self, desc: G.SceneDesc, device: int = 0, td: S.TraversalData | None = None):
        self.desc = desc
        self.device = device
        self.td = td if td is not None else S.build_traversal_data(desc.meshes, desc.instances)
        self.trace_scene = S.DeviceScene(self.td, device)
        sd = ShadingData(desc)
        self.sd = sd
        lib = N.load()
        h = lib.imbart_shading_create(device, N.ptr(sd.vertices), len(sd.vertices), N.ptr(sd.normals),
                                      N.ptr(sd.texcoords), N.ptr(sd.tris), N.ptr(sd.geom_normals), len(sd.tris),
                                      N.ptr(sd.inst_inv), len(sd.inst_inv), N.ptr(sd.mat_kind), N.ptr(sd.mat_params),
                                      len(sd.mat_kind), N.ptr(sd.lights), sd.n_lights, N.ptr(sd.env),
                                      N.ptr(sd.bsphere))
        if not h:
            raise N.ImbartError("imbart_shading_create: " + N.last_error()[1])
        self.shading = h

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

    def __init__(self, scene: GpuScene, max_path_len: int = 10, rr_start: int = 0, max_paths_in_flight: int = 0):
        self.scene = scene
        self.max_path_len = max_path_len
        self.rr_start = rr_start
        self.max_paths = max_paths_in_flight
        lib = N.load()
        self.ctx = lib.imbart_pt_create(scene.device)
        if not self.ctx:
            raise N.ImbartError("imbart_pt_create: " + N.last_error()[1])
        self.last_stats = np.zeros(3, np.int64)

    def render(self, spp: int, seed_base: int, width: int | None = None, height: int | None = None, image=None,
               stream=None, cam: G.Camera | None = None):
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
        stats = np.zeros(3, np.int64)
        N.check(N.load().imbart_pt_render(self.ctx, self.scene.trace_scene.handle, self.scene.shading, N.ptr(r2w),
                                          N.ptr(pos), w, h, spp, self.max_path_len, self.rr_start,
                                          seed_base & (2 ** 64 - 1), N.ptr(image), self.max_paths, N.ptr(stats), st),
                "imbart_pt_render")
        self.last_stats = stats
        return image

    def close(self):
        if getattr(self, "ctx", None):
            N.load().imbart_pt_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
