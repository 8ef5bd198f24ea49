"""Seeded synthetic scenes for the hot path's workloads.

The reference renders OBJ scenes; its own benchmark assets are partly missing and none of
them match the workload sizes this path is measured on, so scenes are generated in memory
from a seed (numpy only). Each generator returns a SceneDesc: meshes, instances, materials,
lights, camera and environment.

  config1  32 displaced icospheres (subdivision 4: 5,120 triangles each, 163,840 total —
           an icosphere at subdivision 4 has 20*4^4 faces), radii U[0.5,2], centres U[-10,10]^3,
           vertices displaced radially by U[-5%,+5%]; a 2-triangle ground quad at y=-10;
           one 2-triangle area light; Lambertian albedo U[0.2,0.8]. One mesh, one instance.
  config2  8 meshes (displaced icospheres and extruded random polygons, 2k-50k triangles)
           instanced 200 times (random rotation, uniform scale U[0.5,3], positions
           U[-10,10]^3): ~1.30M instanced triangles; materials split over Lambertian, Phong,
           Cook-Torrance, glass, mirror; 16 triangular area lights plus a constant environment
           light; a ground quad at y=-13 closes the view (~80% of camera rays hit geometry).
  config3  the config1 generator scaled to ~2M triangles (400 spheres).
  config4  serving: 12 resident scenes of the config1 generator with 10k-2M triangles
           (log-uniform), 256 render requests (scene uniform, pixel count log-uniform in
           [64^2, 1024^2], square, spp in {1, 4, 16, 64}).
  config5  serving under load: Poisson arrivals of progressive 1080p 1-spp increments and
           ray batches of 64k-4M rays (log-uniform; origins uniform in the scene box,
           directions uniform on the sphere) over the config4 scenes.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .scene import Instance, Mesh

# Material kinds (the reference's material classes, render/materials/materials.h, plus the
# Phong class the configs ask for; brdfs.h:48-91 defines the Phong BxDF).
LAMBERT, MIRROR, GLASS, GLOSSY, PHONG, EMISSIVE = 0, 1, 2, 3, 4, 5
# Light kinds besides triangle lights (light.h: DirectionalLight, PointLight, SpotLight).
DIRECTIONAL, POINT, SPOT = 1, 2, 3


@dataclass
class Material:
    kind: int
    color: tuple = (0.8, 0.8, 0.8)          # diffuse albedo / reflectance scale
    specular: tuple = (0.0, 0.0, 0.0)       # glossy/phong specular colour
    exponent: float = 1.0                   # glossy (Blinn) / phong exponent
    eta: float = 1.5                        # glass IOR / mirror eta
    kappa: float = 0.0                      # mirror conductor kappa
    emission: tuple = (0.0, 0.0, 0.0)       # area emitter intensity (emissive faces)
    texture: int = -1                       # diffuse texture (Lambertian, glossy, Phong), index into textures
    bump: int = -1                          # bump map, index into textures


@dataclass
class Camera:
    pos: tuple
    dir: tuple
    up: tuple
    fov: float
    width: int
    height: int


@dataclass
class SceneDesc:
    meshes: list
    instances: list
    materials: list
    lights: list = field(default_factory=list)      # (p0, p1, p2, intensity) per triangle light
    camera: Camera | None = None
    env_intensity: tuple | None = None               # constant environment light
    name: str = ""
    # Lights of the other kinds, after the triangle lights: (kind, 12 floats) with kind
    # DIRECTIONAL (direction of travel, -, -, intensity), POINT (position, -, -, intensity) or
    # SPOT (position, axis, half-angle in radians + 2 unused, intensity).
    delta_lights: list = field(default_factory=list)
    textures: list = field(default_factory=list)     # (height, width, 4) float32 rgba, texel (x, y) at [y, x]
    delta_first: bool = False        # list the delta lights before the triangle lights
    masks: np.ndarray | None = None  # opacity masks per material (MASK_DTYPE), None: all opaque
    mask_buffer: np.ndarray | None = None
    accel_files: list | None = None  # per-mesh acceleration cache files
    env_map: int = -1                # texture index of an environment image (-1: none)
    env_map_intensity: float = 1.0

    @property
    def instanced_triangles(self) -> int:
        return sum(self.meshes[i.mesh_id].triangle_count for i in self.instances)


def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: (V,3) vertices, (F,3) faces; 20*4^level faces."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
                  [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    verts = list(v)
    for _ in range(level):
        cache: dict = {}
        newf = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            newf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(newf, np.int64)
    return np.array(verts, np.float64), f


_ICO_CACHE: dict = {}


def displaced_sphere(rng: np.random.Generator, level: int, center, radius: float, disp: float = 0.05):
    if level not in _ICO_CACHE:
        _ICO_CACHE[level] = icosphere(level)
    v, f = _ICO_CACHE[level]
    scale = radius * (1.0 + rng.uniform(-disp, disp, size=(len(v), 1)))
    return (v * scale + np.asarray(center)).astype(np.float32), f.astype(np.int32)


def extruded_polygon(rng: np.random.Generator, n_sides: int, n_segments: int, height: float = 2.0):
    """Random star-shaped polygon in the xz plane extruded along y, with capped ends."""
    ang = np.sort(rng.uniform(0, 2 * np.pi, n_sides))
    rad = rng.uniform(0.5, 1.0, n_sides)
    ring = np.stack([np.cos(ang) * rad, np.zeros(n_sides), np.sin(ang) * rad], 1)
    ys = np.linspace(-height / 2, height / 2, n_segments + 1)
    verts = np.concatenate([ring + np.array([0, y, 0]) for y in ys])
    faces = []
    for s in range(n_segments):
        a0, b0 = s * n_sides, (s + 1) * n_sides
        for i in range(n_sides):
            j = (i + 1) % n_sides
            faces += [[a0 + i, b0 + i, a0 + j], [a0 + j, b0 + i, b0 + j]]
    # caps: fan around a centre vertex
    for level, flip in ((0, True), (n_segments, False)):
        c = len(verts)
        verts = np.concatenate([verts, [[0, ys[level], 0]]])
        base = level * n_sides
        for i in range(n_sides):
            j = (i + 1) % n_sides
            faces.append([c, base + j, base + i] if flip else [c, base + i, base + j])
    return verts.astype(np.float32), np.array(faces, np.int32)


def quad(p0, p1, p2, p3):
    v = np.array([p0, p1, p2, p3], np.float32)
    f = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    return v, f


def _merge(parts):
    """Merges (verts, faces, material) parts into one Mesh."""
    vs, fs, ms = [], [], []
    off = 0
    for v, f, m in parts:
        vs.append(v)
        fs.append(f + off)
        ms.append(np.full(len(f), m, np.int32))
        off += len(v)
    idx = np.concatenate([np.concatenate(fs), np.concatenate(ms)[:, None]], 1)
    return Mesh(np.concatenate(vs), idx)


def rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _sphere_field(seed: int, n_spheres: int, level: int, width: int, height: int, name: str) -> SceneDesc:
    rng = np.random.default_rng(seed)
    materials: list[Material] = []
    parts = []
    for _ in range(n_spheres):
        c = rng.uniform(-10, 10, 3)
        r = rng.uniform(0.5, 2.0)
        v, f = displaced_sphere(rng, level, c, r)
        materials.append(Material(LAMBERT, color=tuple(rng.uniform(0.2, 0.8, 3))))
        parts.append((v, f, len(materials) - 1))
    materials.append(Material(LAMBERT, color=tuple(rng.uniform(0.2, 0.8, 3))))
    parts.append((*quad([-60, -10, -60], [-60, -10, 60], [60, -10, 60], [60, -10, -60]), len(materials) - 1))
    # Area light: a 2-triangle quad facing down; each emissive face gets its own material
    # (build_scene.cpp:215-233 duplicates the material per emissive face).
    lp = [[-3, 16, -3], [3, 16, -3], [3, 16, 3], [-3, 16, 3]]
    intensity = (40.0, 40.0, 40.0)
    lights = []
    for tri in ([lp[0], lp[1], lp[2]], [lp[0], lp[2], lp[3]]):
        materials.append(Material(EMISSIVE, color=(0.0, 0.0, 0.0), emission=intensity))
        parts.append((np.array(tri, np.float32), np.array([[0, 1, 2]], np.int32), len(materials) - 1))
        lights.append((np.array(tri[0], np.float32), np.array(tri[1], np.float32), np.array(tri[2], np.float32),
                       np.array(intensity, np.float32)))
    mesh = _merge(parts)
    cam = Camera(pos=(0.0, 4.0, -38.0), dir=(0.0, -0.1, 1.0), up=(0.0, 1.0, 0.0), fov=60.0,
                 width=width, height=height)
    return SceneDesc([mesh], [Instance(0)], materials, lights, cam, None, name)


def config1(seed: int = 1, width: int = 512, height: int = 512) -> SceneDesc:
    return _sphere_field(seed, 32, 4, width, height, "config1")


def config3(seed: int = 1, width: int = 1280, height: int = 720) -> SceneDesc:
    return _sphere_field(seed, 400, 4, width, height, "config3")


# Mesh sizes and instance counts of config2: (kind, size parameter, instances).
_C2_MESHES = [("sphere", 4, 40), ("poly", (64, 16), 40), ("poly", (96, 16), 30), ("sphere", 4, 30),
              ("poly", (128, 20), 25), ("poly", (128, 32), 20), ("sphere", 5, 10), ("poly", (384, 64), 5)]


def config2(seed: int = 1, width: int = 1920, height: int = 1080) -> SceneDesc:
    rng = np.random.default_rng(seed)
    meshes: list[Mesh] = []
    materials: list[Material] = []
    # Material class per mesh, balanced by instance count over the five classes.
    classes = [LAMBERT, PHONG, GLOSSY, MIRROR, GLASS, GLASS, MIRROR, GLOSSY]
    for (kind, param, _), cls in zip(_C2_MESHES, classes):
        if kind == "sphere":
            v, f = displaced_sphere(rng, param, (0, 0, 0), 1.0)
        else:
            v, f = extruded_polygon(rng, param[0], param[1])
        if cls == LAMBERT:
            mat = Material(LAMBERT, color=tuple(rng.uniform(0.2, 0.8, 3)))
        elif cls == PHONG:
            mat = Material(PHONG, color=tuple(rng.uniform(0.2, 0.8, 3)), specular=tuple(rng.uniform(0.2, 0.8, 3)),
                           exponent=float(rng.uniform(10, 200)))
        elif cls == GLOSSY:
            # Cook-Torrance roughness r in [0.05, 0.5] mapped to a Blinn exponent 2/r^2 - 2.
            rough = float(rng.uniform(0.05, 0.5))
            mat = Material(GLOSSY, color=tuple(rng.uniform(0.2, 0.8, 3)), specular=tuple(rng.uniform(0.2, 0.8, 3)),
                           exponent=2.0 / rough ** 2 - 2.0)
        elif cls == MIRROR:
            mat = Material(MIRROR, color=(0.9, 0.9, 0.9), eta=0.2, kappa=3.0)
        else:
            mat = Material(GLASS, color=(0.95, 0.95, 0.95), specular=(1.0, 1.0, 1.0), eta=1.5)
        materials.append(mat)
        idx = np.concatenate([f, np.full((len(f), 1), len(materials) - 1, np.int32)], 1)
        meshes.append(Mesh(v, idx))
    instances: list[Instance] = []
    for mesh_id, (_, _, count) in enumerate(_C2_MESHES):
        for _ in range(count):
            m = np.eye(4)
            s = rng.uniform(0.5, 3.0)
            m[:3, :3] = rotation(rng) * s
            m[:3, 3] = rng.uniform(-10, 10, 3)
            instances.append(Instance(mesh_id, m.astype(np.float32)))
    # 16 triangular area lights in one mesh above the field.
    lparts = []
    lights = []
    for i in range(16):
        c = np.array([rng.uniform(-15, 15), 25.0, rng.uniform(-15, 15)])
        p0, p1, p2 = c + [-3, 0, -3], c + [3, 0, -3], c + [0, 0, 3]
        tri = np.array([p0, p2, p1], np.float32)   # facing down
        intensity = np.array(rng.uniform(20, 60, 3), np.float32)
        materials.append(Material(EMISSIVE, color=(0.0, 0.0, 0.0), emission=tuple(intensity)))
        lparts.append((tri, np.array([[0, 1, 2]], np.int32), len(materials) - 1))
        lights.append((tri[0], tri[1], tri[2], intensity))
    # A Lambertian ground quad below the field closes the view (as in config1).
    materials.append(Material(LAMBERT, color=tuple(rng.uniform(0.2, 0.8, 3))))
    lparts.append((*quad([-200, -13, -200], [-200, -13, 200], [200, -13, 200], [200, -13, -200]),
                   len(materials) - 1))
    meshes.append(_merge(lparts))
    instances.append(Instance(len(meshes) - 1))
    cam = Camera(pos=(0.0, 4.0, -30.0), dir=(0.0, -0.12, 1.0), up=(0.0, 1.0, 0.0), fov=50.0,
                 width=width, height=height)
    return SceneDesc(meshes, instances, materials, lights, cam, (0.3, 0.35, 0.4), "config2")


def random_rays(rng: np.random.Generator, n: int, lo, hi, tmin: float = 0.0, tmax: float = 3.0e38) -> np.ndarray:
    """Ray batch: origins uniform in [lo, hi], directions uniform on the sphere."""
    from .native import RAY_DTYPE
    rays = np.zeros(n, RAY_DTYPE)
    org = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["org"][:, :3] = org
    rays["org"][:, 3] = tmin
    rays["dir"][:, :3] = d.astype(np.float32)
    rays["dir"][:, 3] = tmax
    return rays


# ---------------------------------------------------------------------------------------
# Serving workloads
# ---------------------------------------------------------------------------------------
def config4_scene_sizes(n_scenes: int = 12, lo: int = 10_000, hi: int = 2_000_000) -> list[int]:
    """Triangle counts of the resident scenes: log-uniformly spaced from lo to hi."""
    return [int(round(lo * (hi / lo) ** (k / max(n_scenes - 1, 1)))) for k in range(n_scenes)]


def config4_scenes(seed: int = 1, n_scenes: int = 12, lo: int = 10_000, hi: int = 2_000_000) -> list[SceneDesc]:
    """Sphere fields (the config1 generator) with about the requested triangle counts."""
    out = []
    for k, tris in enumerate(config4_scene_sizes(n_scenes, lo, hi)):
        n_spheres = max(1, int(round(tris / 5120)))
        out.append(_sphere_field(seed + 100 * k, n_spheres, 4, 512, 512, f"serve{k}"))
    return out


@dataclass
class RenderJob:
    scene: int
    width: int
    height: int
    spp: int          # samples per pixel (PT) or iterations (BPT, VCM: one camera sample each)
    seed: int
    arrival_s: float = 0.0
    integrator: str = "pt"


@dataclass
class RayJob:
    scene: int
    count: int
    flags: int
    seed: int
    arrival_s: float = 0.0


def config4_requests(seed: int = 1, n: int = 256, n_scenes: int = 12, min_side: int = 64,
                     max_side: int = 1024, mix: tuple = (("pt", 0.7), ("bpt", 0.2), ("vcm", 0.1))) -> list[RenderJob]:
    """All requests arrive at once (a closed batch): square frames with log-uniform sides,
    spp (or iterations) in {1, 4, 16, 64}, integrators drawn from `mix`."""
    rng = np.random.default_rng(seed)
    pick = np.random.default_rng(seed + 1000)
    names, probs = [m[0] for m in mix], np.array([m[1] for m in mix], np.float64)
    jobs = []
    for i in range(n):
        side = int(round(np.exp(rng.uniform(np.log(min_side), np.log(max_side)))))
        jobs.append(RenderJob(int(rng.integers(n_scenes)), side, side, int(rng.choice([1, 4, 16, 64])),
                              int(rng.integers(1, 2 ** 31)),
                              integrator=names[int(pick.choice(len(names), p=probs / probs.sum()))]))
    return jobs


def config5_requests(seed: int = 1, rate: float = 100.0, duration_s: float = 4.0, n_scenes: int = 12,
                     ray_share: float = 0.5, min_rays: int = 65536, max_rays: int = 4 << 20,
                     width: int = 1920, height: int = 1080) -> list:
    """Poisson arrivals at `rate` requests/s for `duration_s`: 1-spp frames of width x height
    (a progressive increment: its own seed) or ray batches (closest-hit and any-hit alike)."""
    rng = np.random.default_rng(seed)
    t, jobs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            break
        scene = int(rng.integers(n_scenes))
        if rng.uniform() < ray_share:
            count = int(round(np.exp(rng.uniform(np.log(min_rays), np.log(max_rays)))))
            jobs.append(RayJob(scene, count, int(rng.integers(2)), int(rng.integers(1, 2 ** 31)), t))
        else:
            jobs.append(RenderJob(scene, width, height, 1, int(rng.integers(1, 2 ** 31)), t))
    return jobs


def scene_box(desc: SceneDesc) -> tuple[np.ndarray, np.ndarray]:
    """World-space box of a scene's instanced meshes."""
    lo = np.full(3, np.inf, np.float32)
    hi = np.full(3, -np.inf, np.float32)
    for inst in desc.instances:
        mlo, mhi = desc.meshes[inst.mesh_id].bounding_box()
        m = inst.mat[:3, :]
        c = m[:, :3] @ ((mhi + mlo) * np.float32(0.5)) + m[:, 3]
        e = np.abs(m[:, :3]) @ ((mhi - mlo) * np.float32(0.5))
        lo = np.minimum(lo, c - e)
        hi = np.maximum(hi, c + e)
    return lo, hi
