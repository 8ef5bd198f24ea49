"""Directional, point and spot lights, diffuse textures and bump maps against the reference.

The scene mixes every light kind of the reference (environment, triangle, directional,
point, spot), a textured Lambertian sphere and ground, a textured Phong sphere and bump maps
on a glossy and a mirror sphere. Path-traced images are compared with the reference's
PathTracer (rel. RMSE 1e-3, as for the other path-tracer tests); the VCM family's light and
camera passes with the reference's VCMIntegrator as in test_vcm.py.
"""
import numpy as np
import pytest

from imbatracer_b200 import scenegen as G
from oracle import refwrap as R
from tests import test_vcm as V
from tests.test_pt import small_mixed_scene

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference tree absent)")

RMSE_TOL = 1e-3


def rel_rmse(a, b):
    den = np.sqrt(np.mean(b.astype(np.float64) ** 2))
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) / max(den, 1e-30))


def checker(w, h, a, b, cells=4):
    y, x = np.mgrid[0:h, 0:w]
    on = ((x * cells // w) + (y * cells // h)) % 2 == 0
    img = np.where(on[..., None], np.array(a + (1.0,), np.float32), np.array(b + (1.0,), np.float32))
    return np.ascontiguousarray(img.astype(np.float32))


def bumps(w, h):
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    v = 0.5 + 0.5 * np.sin(x * 0.7) * np.cos(y * 0.5)
    return np.ascontiguousarray(np.stack([v, v, v, np.ones_like(v)], -1).astype(np.float32))


def lit_textured_scene():
    d = small_mixed_scene()
    # Spherical texcoords on the spheres (outside [0, 1] and negative, to exercise wrapping),
    # planar ones on the ground-and-lights mesh.
    for m in d.meshes[:-1]:
        v = m.vertices - m.vertices.mean(0)
        r = np.linalg.norm(v, axis=1, keepdims=True)
        u = np.arctan2(v[:, 2], v[:, 0]) / np.pi * 1.5
        t = np.arccos(np.clip(v[:, 1:2] / r, -1, 1))[:, 0] / np.pi * 2.0 - 0.5
        m.texcoords = np.stack([u, t], 1).astype(np.float32)
    g = d.meshes[-1]
    g.texcoords = np.stack([g.vertices[:, 0] / 7.0, g.vertices[:, 2] / 5.0], 1).astype(np.float32)
    d.textures = [checker(16, 8, (0.8, 0.2, 0.2), (0.2, 0.6, 0.9)), bumps(32, 32),
                  checker(8, 8, (0.9, 0.9, 0.3), (0.1, 0.1, 0.1), cells=2)]
    d.materials[0].texture = 0          # Lambertian sphere: checker
    d.materials[1].texture = 2          # Phong sphere: diffuse texture
    d.materials[2].bump = 1             # glossy sphere: bump map
    d.materials[3].bump = 1             # mirror: bump map
    d.materials[5].texture = 2          # ground
    n = lambda v: (np.asarray(v, np.float32) / np.linalg.norm(v)).tolist()
    d.delta_lights = [
        (G.DIRECTIONAL, n([0.3, -1.0, 0.2]) + [0.0] * 6 + [1.2, 1.1, 1.0]),
        (G.POINT, [2.0, 3.5, -3.0] + [0.0] * 6 + [60.0, 55.0, 50.0]),
        (G.SPOT, [-3.0, 5.0, -2.0] + n([0.2, -1.0, 0.3]) + [0.45, 0.0, 0.0] + [90.0, 85.0, 95.0]),
    ]
    d.name = "lit_textured"
    return d


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("w,h,spp,max_len,seed", [(96, 64, 6, 6, 4242), (48, 32, 3, 3, 77)])
def test_path_tracer_with_all_light_kinds_and_textures(cuda, w, h, spp, max_len, seed):
    from imbatracer_b200.integrators import GpuScene, PathTracer
    d = lit_textured_scene()
    ref = R.RefScene(d).render_pt(w, h, spp, max_len, seed)
    gs = GpuScene(d)
    img = PathTracer(gs, max_path_len=max_len).render(spp, seed, w, h).cpu().numpy()
    assert ref.sum() > 0
    err = rel_rmse(img, ref)
    assert err <= RMSE_TOL, err


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("algo", ["vcm", "bpt", "lt"])
def test_light_pass_with_all_light_kinds_and_textures(cuda, algo):
    from imbatracer_b200.integrators import GpuScene
    d = lit_textured_scene()
    rv = R.RefVcm(R.RefScene(d), algo, V.W, V.Hh, max_path_len=V.MAX_LEN, light_path_count=V.LIGHT_PATHS)
    rv.begin_iteration(1)
    ref_img = rv.light_pass(321, 17)
    ref_v = rv.light_vertices()
    gs = GpuScene(d)
    vi = V.gpu_integrator(gs, algo, rv)
    vi.begin_iteration(1)
    img = vi.light_pass(321, 17).cpu().numpy()
    got_v = vi.light_vertices()
    if algo != "lt":
        assert len(ref_v) > 100 and abs(len(got_v) - len(ref_v)) <= max(2, 0.01 * len(ref_v))
        ok, _ = V.match_vertices(ref_v, got_v)
        assert ok.mean() >= V.MATCH_MIN, ok.mean()
    assert ref_img.sum() > 0
    assert rel_rmse(img, ref_img) <= V.LIGHT_IMAGE_TOL


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("algo", ["vcm", "bpt", "ppm", "pt"])
def test_camera_pass_with_all_light_kinds_and_textures(cuda, algo):
    from imbatracer_b200.integrators import GpuScene
    d = lit_textured_scene()
    rv = R.RefVcm(R.RefScene(d), algo, V.W, V.Hh, max_path_len=V.MAX_LEN, light_path_count=V.LIGHT_PATHS)
    gs = GpuScene(d)
    vi = V.gpu_integrator(gs, algo, rv)
    rv.begin_iteration(1)
    rv.light_pass(555, 3)
    ref_v = rv.light_vertices()
    ref = rv.camera_pass(666)
    vi.begin_iteration(1)
    vi.load_light_vertices(ref_v)
    img = vi.camera_pass(666).cpu().numpy()
    assert ref.sum() > 0
    assert rel_rmse(img, ref) <= V.IMAGE_TOL
