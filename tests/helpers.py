"""Shared fixtures-as-functions for the parity tests (scenes, ray sets, comparisons)."""
from __future__ import annotations

import functools

import numpy as np

from imbatracer_b200 import native as N
from imbatracer_b200 import scene as S
from imbatracer_b200 import scenegen as G


@functools.lru_cache(maxsize=None)
def scene_desc(name: str):
    if name == "config1":
        return G.config1()
    if name == "config2":
        return G.config2()
    if name == "tiny":
        return tiny_scene()
    raise KeyError(name)


@functools.lru_cache(maxsize=None)
def traversal_data(name: str):
    d = scene_desc(name)
    return S.build_traversal_data(d.meshes, d.instances)


def tiny_scene():
    """A handful of triangles: shared edges, a degenerate triangle, an axis-aligned quad, and
    two instances of a single-triangle mesh (the single-leaf root wrapper)."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0],         # two triangles sharing an edge
                  [0, 0, 2], [2, 0, 2], [0, 2, 2],                     # a parallel triangle behind
                  [3, 3, 3], [3, 3, 3], [3, 3, 3]], np.float32)        # a degenerate triangle
    idx = np.array([[0, 1, 2, 0], [1, 3, 2, 0], [4, 5, 6, 1], [7, 8, 9, 1]], np.int32)
    m0 = S.Mesh(v, idx)
    m1 = S.Mesh(np.array([[-1, -1, 5], [1, -1, 5], [0, 1, 5]], np.float32), np.array([[0, 1, 2, 2]], np.int32))
    t = np.eye(4, dtype=np.float32)
    t[:3, 3] = [0.5, 0.5, 1.0]
    r = np.eye(4, dtype=np.float32)
    r[:3, :3] = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], np.float32) * 2.0
    insts = [S.Instance(0), S.Instance(1), S.Instance(1, t), S.Instance(1, r)]
    return G.SceneDesc([m0, m1], insts, [G.Material(G.LAMBERT)] * 3, name="tiny")


def ray_set(name: str, n: int, seed: int = 0) -> np.ndarray:
    """Random rays through the scene's bounds plus rays aimed at triangle vertices, edges
    and centroids (the watertightness and tie cases), plus invalid/padding rays."""
    rng = np.random.default_rng(seed)
    d = scene_desc(name)
    allv = []
    for inst in d.instances:
        m = d.meshes[inst.mesh_id]
        allv.append(m.vertices @ inst.mat[:3, :3].T + inst.mat[:3, 3])
    allv = np.concatenate(allv)
    lo, hi = allv.min(0), allv.max(0)
    ext = hi - lo
    n_rand = n // 2
    rays = G.random_rays(rng, n_rand, lo - 0.1 * ext, hi + 0.1 * ext)
    # Rays aimed at vertices / edge midpoints / centroids of random instanced triangles.
    n_aim = n - n_rand - 16
    targets = []
    for _ in range(n_aim):
        inst = d.instances[rng.integers(len(d.instances))]
        m = d.meshes[inst.mesh_id]
        t = m.indices[rng.integers(m.triangle_count), :3]
        p = m.vertices[t].astype(np.float64)
        kind = rng.integers(3)
        if kind == 0:
            q = p[rng.integers(3)]
        elif kind == 1:
            q = 0.5 * (p[0] + p[1])
        else:
            q = p.mean(0)
        targets.append(inst.mat[:3, :3].astype(np.float64) @ q + inst.mat[:3, 3])
    targets = np.array(targets).reshape(-1, 3)
    org = rng.uniform(lo - 0.5 * ext, hi + 0.5 * ext, size=(len(targets), 3))
    dirs = targets - org
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    aim = np.zeros(len(targets), N.RAY_DTYPE)
    aim["org"][:, :3] = org
    aim["dir"][:, :3] = dirs
    aim["dir"][:, 3] = 3.0e38
    # Edge cases: zero rays (queue padding), empty interval, tmin > 0, axis-aligned directions.
    edge = np.zeros(16, N.RAY_DTYPE)
    c = 0.5 * (lo + hi)
    edge["org"][4:, :3] = c
    edge["dir"][4:8, 3] = 1.0e30
    edge["dir"][4, :3] = [1, 0, 0]
    edge["dir"][5, :3] = [0, -1, 0]
    edge["dir"][6, :3] = [0, 0, 1]
    edge["dir"][7, :3] = [0, 0, -1]
    edge["dir"][8:12, :3] = [0.3, -0.8, 0.2]
    edge["dir"][8:12, 3] = [1e30, 5.0, 0.5, 0.0]     # bounded tmax, including tmax == tmin
    edge["org"][12:16, 3] = [0.1, 1.0, 10.0, 2e30]   # tmin > 0, tmin > tmax for the last
    edge["dir"][12:16, :3] = [-0.2, -0.9, 0.4]
    edge["dir"][12:16, 3] = 1e30
    return np.concatenate([rays, aim, edge])


def hits_equal(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-ray bitwise equality of hit records."""
    return (a.view(np.int32).reshape(-1, 4) == b.view(np.int32).reshape(-1, 4)).all(1)


def wide_arrays(td, node_width=None):
    """Host-side wide conversion of a traversal data set (no GPU), 8-wide unless node_width
    says 4."""
    from oracle import oracle as O
    lib = N.load()
    prev = lib.imbart_get_node_width()
    if node_width is not None:
        N.check(lib.imbart_set_node_width(node_width), "imbart_set_node_width")
    try:
        cnt = np.zeros(4, np.int32)
        args = (td.root, N.ptr(td.nodes), len(td.nodes), N.ptr(td.instances), len(td.instances), N.ptr(td.tris),
                len(td.tris))
        N.check(lib.imbart_wide_from_node2(*args, None, 0, None, 0, None, 0, N.ptr(cnt)), "wide")
        wn = np.zeros(cnt[0], O.WNODE_DTYPE)
        wt = np.zeros(cnt[1], O.WTRI_DTYPE)
        wi = np.zeros(cnt[2], O.WINST_DTYPE)
        N.check(lib.imbart_wide_from_node2(*args, N.ptr(wn), len(wn), N.ptr(wt), len(wt), N.ptr(wi), len(wi),
                                           N.ptr(cnt)), "wide")
    finally:
        lib.imbart_set_node_width(prev)
    return wn, wt, wi, int(cnt[3])
