"""Python access to the oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and
only as the checker or the timed CPU baseline; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

WNODE_DTYPE = np.dtype([("px", "<f4"), ("py", "<f4"), ("pz", "<f4"), ("ex", "u1"), ("ey", "u1"),
                        ("ez", "u1"), ("imask", "u1"), ("child_base", "<u4"), ("prim_base", "<u4"),
                        ("meta", "u1", 8), ("qlo_x", "u1", 8), ("qhi_x", "u1", 8), ("qlo_y", "u1", 8),
                        ("qhi_y", "u1", 8), ("qlo_z", "u1", 8), ("qhi_z", "u1", 8)])
WTRI_DTYPE = np.dtype([("v0", "<f4", 3), ("id", "<i4"), ("v1", "<f4", 3), ("p0", "<i4"), ("v2", "<f4", 3),
                       ("p1", "<i4")])
WINST_DTYPE = np.dtype([("m", "<f4", 12), ("id", "<i4"), ("root", "<i4"), ("pad", "<i4", 2)])
assert WNODE_DTYPE.itemsize == 80 and WTRI_DTYPE.itemsize == 48 and WINST_DTYPE.itemsize == 64


class Grid(C.Structure):
    _fields_ = [("lo", C.c_float * 3), ("hi", C.c_float * 3), ("radius", C.c_float), ("radius_sqr", C.c_float),
                ("cell_size", C.c_float), ("inv_cell_size", C.c_float), ("table_size", C.c_uint32),
                ("n", C.c_int32)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        P, I = C.c_void_p, C.c_int
        sig = {
            "oracle_trace_node2": (None, [I, P, P, P, P, P, P, I, P, P, P, P, I, I, I]),
            "oracle_trace_brute": (None, [P, P, P, P, P, P, I, P, P, P, I, I, I]),
            "oracle_wide_walk": (None, [P, P, P, I, P, P, P, P, I, I, I, I]),
            "oracle_hashgrid_build": (None, [P, I, I, C.c_float, C.c_float, I, C.POINTER(Grid), P, P]),
            "oracle_hashgrid_query": (None, [C.POINTER(Grid), P, P, P, I, P, I, I, P, P, P, I]),
            "oracle_mwc64x": (C.c_uint32, [P]),
            "oracle_random_float": (C.c_float, [P]),
            "oracle_random_int": (I, [P, I, I]),
            "oracle_seed_state": (C.c_uint64, [C.c_uint64, I, I]),
            "oracle_seed_camera": (None, [C.c_uint64, I, I, I, P]),
            "oracle_draw_floats": (None, [P, I, I, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _lib = lib
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags.c_contiguous, "arrays passed to the oracle must be contiguous"
    return a.ctypes.data


def threads() -> int:
    return os.cpu_count() or 1


def trace_node2(td, rays: np.ndarray, any_hit: bool = False, nthreads: int | None = None, with_v: bool = False):
    """Closest/any hit over a scene's reference-layout traversal data (scene.TraversalData)."""
    from imbatracer_b200.native import HIT_DTYPE
    hits = np.zeros(len(rays), HIT_DTYPE)
    v = np.zeros(len(rays), np.float32) if with_v else None
    masked = td.masks is not None and (np.any(td.masks["width"] * td.masks["height"] != 1) or
                                       np.any(td.mask_buffer[td.masks["offset"]] == 0))
    load().oracle_trace_node2(td.root, _p(td.nodes), _p(td.instances), _p(td.tris),
                              _p(td.indices) if masked else None, _p(td.texcoords) if masked else None,
                              _p(td.masks) if masked else None, len(td.masks) if masked else 0,
                              _p(td.mask_buffer) if masked else None, _p(rays), _p(hits), _p(v), len(rays),
                              1 if any_hit else 0, nthreads or threads())
    return (hits, v) if with_v else hits


def trace_brute(meshes, instances, tri_layout, rays: np.ndarray, any_hit: bool = False, with_v: bool = False):
    """Brute-force closest/any hit over every triangle of every instance."""
    from imbatracer_b200.native import HIT_DTYPE
    tri_arrays, ids, first, count = [], [], [], []
    off = 0
    for mi, m in enumerate(meshes):
        v = m.vertices[m.indices[:, :3]].reshape(-1, 9)
        tri_arrays.append(v)
        ids.append(np.arange(m.triangle_count, dtype=np.int32) + tri_layout[mi])
        first.append(off)
        count.append(m.triangle_count)
        off += m.triangle_count
    mesh_tris = np.ascontiguousarray(np.concatenate(tri_arrays).astype(np.float32))
    mesh_ids = np.ascontiguousarray(np.concatenate(ids))
    first = np.array(first, np.int32)
    count = np.array(count, np.int32)
    inv = np.ascontiguousarray(np.stack([i.inv_mat.reshape(-1) for i in instances]).astype(np.float32))
    inst_mesh = np.array([i.mesh_id for i in instances], np.int32)
    hits = np.zeros(len(rays), HIT_DTYPE)
    vv = np.zeros(len(rays), np.float32) if with_v else None
    load().oracle_trace_brute(_p(mesh_tris), _p(mesh_ids), _p(first), _p(count), _p(inv), _p(inst_mesh),
                              len(instances), _p(rays), _p(hits), _p(vv), len(rays), 1 if any_hit else 0, threads())
    return (hits, vv) if with_v else hits


def wide_walk(wnodes, wtris, winsts, root, rays: np.ndarray, any_hit: bool = False, nthreads: int | None = None):
    """Restatement of the GPU kernel's walk over the 8-wide layout: (hits, bytes per ray,
    [nodes visited, triangles tested, instances entered])."""
    from imbatracer_b200.native import HIT_DTYPE
    hits = np.zeros(len(rays), HIT_DTYPE)
    nbytes = np.zeros(len(rays), np.int64)
    counts = np.zeros(3, np.int64)
    load().oracle_wide_walk(_p(wnodes), _p(wtris), _p(winsts), root, _p(rays), _p(hits), _p(nbytes), _p(counts),
                            len(rays), 1 if any_hit else 0, nthreads or threads(), len(winsts))
    return hits, nbytes, counts


def hashgrid_build(pos: np.ndarray, radius: float, cell_factor: float = 2.0, table_size: int | None = None):
    """Builds the oracle hash grid; returns (Grid, cell_ends, sorted_ids)."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    ts = table_size if table_size is not None else 2 * n
    g = Grid()
    ends = np.zeros(ts, np.int32)
    ids = np.zeros(max(n, 1), np.int32)
    load().oracle_hashgrid_build(_p(pos), pos.shape[1], n, radius, cell_factor, ts, C.byref(g), _p(ends), _p(ids))
    return g, ends, ids


def hashgrid_query(grid, ends, ids, pos: np.ndarray, queries: np.ndarray, k: int, nthreads: int | None = None):
    """k-capped radius query; returns (ids (nq,k) with -1 padding, counts (nq,), d2 (nq,k))."""
    pos = np.ascontiguousarray(pos, np.float32)
    q = np.ascontiguousarray(queries, np.float32)
    out = np.zeros((len(q), k), np.int32)
    cnt = np.zeros(len(q), np.int32)
    d2 = np.zeros((len(q), k), np.float32)
    load().oracle_hashgrid_query(C.byref(grid), _p(ends), _p(ids), _p(pos), pos.shape[1], _p(q), len(q), k,
                                 _p(out), _p(cnt), _p(d2), nthreads or threads())
    return out, cnt, d2


def seed_camera(seed_base: int, first: int, count: int, spp: int) -> np.ndarray:
    st = np.zeros(count, np.uint64)
    load().oracle_seed_camera(seed_base, first, count, spp, _p(st))
    return st


def draw_floats(states: np.ndarray, n: int) -> np.ndarray:
    st = np.ascontiguousarray(states.copy(), np.uint64)
    out = np.zeros((len(st), n), np.float32)
    load().oracle_draw_floats(_p(st), len(st), n, _p(out))
    return out
