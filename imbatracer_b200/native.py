"""ctypes bindings of libimbart's C ABI (include/imbart.h).

The library is the product; this module only loads it and declares the signatures. It
raises immediately when the library is missing: there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

# --- numpy views of the boundary structs (byte layouts of include/imbart.h) -------------
RAY_DTYPE = np.dtype([("org", "<f4", 4), ("dir", "<f4", 4)])
HIT_DTYPE = np.dtype([("tri_id", "<i4"), ("inst_id", "<i4"), ("tmax", "<f4"), ("u", "<f4")])
BBOX_DTYPE = np.dtype([("lo_x", "<f4"), ("hi_x", "<f4"), ("lo_y", "<f4"), ("hi_y", "<f4"),
                       ("lo_z", "<f4"), ("hi_z", "<f4")])
NODE2_DTYPE = np.dtype([("left_bb", BBOX_DTYPE), ("right_bb", BBOX_DTYPE), ("left", "<i4"),
                        ("right", "<i4"), ("pad", "<i4", 2)])
NODE4_DTYPE = np.dtype([("min_x", "<f4", 4), ("max_x", "<f4", 4), ("min_y", "<f4", 4),
                        ("max_y", "<f4", 4), ("min_z", "<f4", 4), ("max_z", "<f4", 4),
                        ("children", "<i4", 4)])
INST_DTYPE = np.dtype([("transf", "<f4", 12), ("id", "<i4"), ("next", "<i4"), ("pad", "<i4", 2)])
MASK_DTYPE = np.dtype([("width", "<i4"), ("height", "<i4"), ("offset", "<i4")])
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16
assert NODE2_DTYPE.itemsize == 64 and NODE4_DTYPE.itemsize == 112 and INST_DTYPE.itemsize == 64

TRACE_CLOSEST = 0
TRACE_ANY = 1
TRACE_COHERENT = 2


class SceneInfo(C.Structure):
    _fields_ = [("wide_nodes", C.c_int64), ("top_nodes", C.c_int64), ("triangles", C.c_int64),
                ("instances", C.c_int64), ("device_bytes", C.c_int64), ("root", C.c_int32),
                ("masked", C.c_int32), ("node_width", C.c_int32), ("reserved", C.c_int32)]


class PtProfile(C.Structure):
    _fields_ = [("events", C.c_int), ("work", C.c_int), ("closest_ms", C.c_double), ("shadow_ms", C.c_double),
                ("closest_launches", C.c_longlong), ("shadow_launches", C.c_longlong),
                ("closest_rays", C.c_longlong), ("shadow_rays", C.c_longlong),
                ("closest_work", C.c_ulonglong * 3), ("shadow_work", C.c_ulonglong * 3)]


class Camera(C.Structure):
    _fields_ = [("raster_to_world", C.c_float * 16), ("world_to_raster", C.c_float * 16), ("pos", C.c_float * 3),
                ("dir", C.c_float * 3), ("img_plane_dist", C.c_float), ("width", C.c_int), ("height", C.c_int)]


class VcmSettings(C.Structure):
    _fields_ = [("algorithm", C.c_int), ("spp", C.c_int), ("max_path_len", C.c_int), ("light_path_count", C.c_int),
                ("num_connections", C.c_int), ("num_knn", C.c_int), ("light_tile_size", C.c_int),
                ("base_radius", C.c_float), ("light_seed", C.c_ulonglong), ("light_seed_step", C.c_ulonglong),
                ("camera_seed", C.c_ulonglong), ("radius_exponent", C.c_float), ("grid_cell_factor", C.c_float),
                ("grid_table_size", C.c_int)]


VCM, BPT, PPM, LT, VCM_PT = 0, 1, 2, 3, 4
ACCEL_GPU, ACCEL_CPU = 1, 2   # block types of the acceleration cache files

VCM_ALGORITHMS = {"vcm": VCM, "bpt": BPT, "ppm": PPM, "lt": LT, "pt": VCM_PT}


class SceneSource(C.Structure):
    _fields_ = [("root", C.c_int), ("nodes", C.c_void_p), ("n_nodes", C.c_int),
                ("instances", C.c_void_p), ("n_instances", C.c_int), ("tris", C.c_void_p), ("n_tri_vec4", C.c_int),
                ("vertices", C.c_void_p), ("n_vertices", C.c_int), ("normals", C.c_void_p), ("texcoords", C.c_void_p),
                ("mesh_tris", C.c_void_p), ("geom_normals", C.c_void_p), ("n_mesh_tris", C.c_int),
                ("inst_inv", C.c_void_p), ("n_inst_inv", C.c_int), ("mat_kind", C.c_void_p),
                ("mat_params", C.c_void_p), ("n_mats", C.c_int), ("tri_lights", C.c_void_p), ("n_tri_lights", C.c_int),
                ("env_color", C.c_void_p), ("bsphere", C.c_void_p), ("light_kinds", C.c_void_p),
                ("tex_dims", C.c_void_p), ("tex_pixels", C.c_void_p), ("n_textures", C.c_int),
                ("env_map", C.c_int), ("env_intensity", C.c_float)]


class TraceTuning(C.Structure):
    _fields_ = [("variant", C.c_int), ("refill", C.c_int), ("ms", C.c_float), ("default_ms", C.c_float),
                ("tri_batch", C.c_int)]


class MeshDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("n_vertices", C.c_int), ("indices", C.c_void_p), ("n_tris", C.c_int),
                ("tri_offset", C.c_int)]


class InstanceDesc(C.Structure):
    _fields_ = [("obj_to_world", C.c_float * 12), ("world_to_obj", C.c_float * 12), ("mesh", C.c_int),
                ("id", C.c_int)]


class VcmRequest(C.Structure):
    _fields_ = [("scene", C.c_int), ("camera", Camera), ("settings", VcmSettings), ("radius_factor", C.c_float),
                ("iterations", C.c_int), ("seed_step", C.c_ulonglong), ("image_host", C.c_void_p)]


class RenderRequest(C.Structure):
    _fields_ = [("scene", C.c_int), ("raster_to_world", C.c_float * 16), ("cam_pos", C.c_float * 3),
                ("width", C.c_int), ("height", C.c_int), ("spp", C.c_int), ("max_path_len", C.c_int),
                ("rr_start", C.c_int), ("seed_base", C.c_ulonglong), ("image_host", C.c_void_p)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("kind", C.c_int), ("submit_ms", C.c_double), ("start_ms", C.c_double),
                ("done_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in ("submitted", "completed", "failed", "waves", "closest_rays", "shadow_rays",
                                            "batch_rays", "scene_uploads", "scene_evictions", "pool_bytes",
                                            "pool_used_bytes", "kernel_launches")]


SERVE_BATCHED = 0
SERVE_PLAIN = 1


class ImbartError(RuntimeError):
    pass


_lib = None

P = C.c_void_p
I = C.c_int

# name -> (restype, argtypes)
_SIGNATURES = {
    "imbart_last_error": (I, []),
    "imbart_last_error_string": (C.c_char_p, []),
    "imbart_clear_error": (None, []),
    "imbart_version": (C.c_char_p, []),
    "imbart_invalidate_scenes": (None, []),
    "imbart_scene_from_node2": (P, [I, P, I, P, I, P, I, P, I, P, I, P, I, P, I, I]),
    "imbart_scene_from_node4": (P, [I, P, I, P, I, P, I, P, I, P, I, P, I, P, I, I]),
    "imbart_scene_destroy": (None, [P]),
    "imbart_wide_from_node2": (I, [I, P, I, P, I, P, I, P, I, P, I, P, I, P]),
    "imbart_set_node_width": (I, [I]),
    "imbart_get_node_width": (I, []),
    "imbart_scene_get_info": (I, [P, C.POINTER(SceneInfo)]),
    "imbart_scene_get_device_arrays": (I, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "imbart_trace": (I, [P, P, P, I, I, P]),
    "imbart_trace_uv": (I, [P, P, P, P, I, I, P]),
    "imbart_trace_host": (I, [P, P, P, I, I, P]),
    "imbart_trace_stats": (I, [P, P, P, I, I, P, P]),
    "imbart_scene_error_count": (I, [P]),
    "imbart_kernel_launch_count": (C.c_int64, []),
    "imbart_hashgrid_create": (P, [I]),
    "imbart_hashgrid_destroy": (None, [P]),
    "imbart_hashgrid_build": (I, [P, P, I, I, C.c_float, C.c_float, I, P]),
    "imbart_hashgrid_query": (I, [P, P, I, I, P, P, P, P]),
    "imbart_hashgrid_build_host": (I, [P, P, I, I, C.c_float, C.c_float, I]),
    "imbart_hashgrid_query_host": (I, [P, P, I, I, P, P, P]),
    "imbart_hashgrid_get_params": (I, [P, P, P, P]),
    "imbart_hashgrid_get_arrays": (I, [P, C.POINTER(P), C.POINTER(P)]),
    "imbart_hashgrid_build_noalloc": (I, [P, I, I, C.c_float, C.c_float, I, P, P, P, P]),
    "imbart_camera_setup": (I, [P, P, P, C.c_float, C.c_float, C.c_float, C.c_float, P, P, P]),
    "imbart_camera_rays": (I, [P, P, I, I, I, C.c_uint64, C.c_longlong, I, P, P, P, P, P]),
    "imbart_shading_create": (P, [I, P, I, P, P, P, P, I, P, I, P, P, I, P, I, P, P]),
    "imbart_shading_destroy": (None, [P]),
    "imbart_shading_create_ex": (P, [I, P, I, P, P, P, P, I, P, I, P, P, I, P, P, I, P, P, P, P, I]),
    "imbart_pt_create": (P, [I]),
    "imbart_pt_destroy": (None, [P]),
    "imbart_pt_render": (I, [P, P, P, P, P, I, I, I, I, I, C.c_uint64, P, C.c_longlong, P, P]),
    "imbart_pt_render_range": (I, [P, P, P, P, P, I, I, I, I, I, C.c_uint64, P, C.c_longlong, C.c_longlong,
                                   C.c_longlong, P, P]),
    "imbart_pt_set_profile": (I, [P, P]),
    "imbart_pt_set_graphs": (I, [P, I]),
    "imbart_group_by_key": (I, [P, I, P, P]),
    "imbart_set_trace_config": (I, [I, I, I]),
    "imbart_get_trace_config": (I, [C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
    "imbart_set_trace_variant_any": (I, [I]),
    "imbart_get_trace_variant_any": (I, []),
    "imbart_build_mesh_node2": (I, [P, I, I, P, I, I, I, P, I, P, P, I, P]),
    "imbart_build_mesh_node2_ex": (I, [P, I, I, P, I, I, I, C.c_float, P, I, P, P, I, P]),
    "imbart_accel_file_info": (I, [C.c_char_p, I, P, P]),
    "imbart_set_trace_class": (I, [I, I, I]),
    "imbart_get_trace_class": (I, [I, P, P]),
    "imbart_trace_autotune": (I, [P, P, P, I, I, P, C.POINTER(TraceTuning)]),
    "imbart_set_trace_tri_batch": (I, [I, I]),
    "imbart_get_trace_tri_batch": (I, [I]),
    "imbart_shading_set_env_map": (I, [P, I, C.c_float]),
    "imbart_scene_build_gpu": (P, [C.POINTER(MeshDesc), I, C.POINTER(InstanceDesc), I, I, P, C.POINTER(C.c_float)]),
    "imbart_scene_refit": (I, [P, P, C.c_longlong, P, I, P]),
    "imbart_load_accel_node2": (I, [C.c_char_p, I, P, I, P, P, I, P]),
    "imbart_load_accel_node4": (I, [C.c_char_p, I, P, I, P, P, I, P]),
    "imbart_store_accel_node2": (I, [C.c_char_p, P, I, I, P, I, I, I]),
    "imbart_store_accel_node4": (I, [C.c_char_p, P, I, I, P, I, I, I]),
    "imbart_build_top_node2": (I, [P, P, P, I, P, I, P, P]),
    "imbart_camera_make": (I, [P, P, P, C.c_float, I, I, C.POINTER(Camera)]),
    "imbart_estimate_pixel_size": (I, [P, C.POINTER(Camera), P, P]),
    "imbart_vcm_create": (P, [I]),
    "imbart_vcm_destroy": (None, [P]),
    "imbart_vcm_begin_iteration": (I, [P, C.POINTER(VcmSettings), I, P]),
    "imbart_vcm_light_pass": (I, [P, P, P, C.POINTER(Camera), C.POINTER(VcmSettings), P, P, P]),
    "imbart_vcm_camera_pass": (I, [P, P, P, C.POINTER(Camera), C.POINTER(VcmSettings), P, C.c_longlong, P, P]),
    "imbart_vcm_light_pass_range": (I, [P, P, P, C.POINTER(Camera), C.POINTER(VcmSettings), I, I, P, P, I, P, P]),
    "imbart_vcm_camera_pass_range": (I, [P, P, P, C.POINTER(Camera), C.POINTER(VcmSettings), C.c_longlong,
                                         C.c_longlong, P, C.c_longlong, P, P]),
    "imbart_vcm_render": (I, [P, P, P, C.POINTER(Camera), C.POINTER(VcmSettings), I, P, C.c_longlong, P, P]),
    "imbart_vcm_light_vertices": (I, [P, C.POINTER(P), C.POINTER(I)]),
    "imbart_vcm_copy_light_vertices": (I, [P, P, I]),
    "imbart_vcm_load_light_vertices": (I, [P, C.POINTER(VcmSettings), P, I, P]),
    "imbart_server_create": (P, [I, I, C.c_longlong, C.c_longlong]),
    "imbart_server_destroy": (None, [P]),
    "imbart_server_add_scene": (I, [P, C.POINTER(SceneSource)]),
    "imbart_server_add_scene_gpu_build": (I, [P, P, C.POINTER(MeshDesc), I, C.POINTER(InstanceDesc), I, C.POINTER(C.c_float)]),
    "imbart_server_submit_render": (C.c_longlong, [P, C.POINTER(RenderRequest)]),
    "imbart_server_submit_rays": (C.c_longlong, [P, I, P, P, I, I]),
    "imbart_server_submit_vcm": (C.c_longlong, [P, C.POINTER(VcmRequest)]),
    "imbart_server_wait": (I, [P, C.c_longlong, C.POINTER(RequestResult)]),
    "imbart_server_drain": (I, [P]),
    "imbart_server_get_stats": (I, [P, C.POINTER(ServerStats)]),
    "intersect_gpu_masked_instanced": (None, [I, P, P, P, P, P, P, P, P, P, I]),
    "occluded_gpu_masked_instanced": (None, [I, P, P, P, P, P, P, P, P, P, I]),
    "intersect_cpu_masked_instanced": (None, [I, P, P, P, P, P, P, P, P, P, I]),
    "occluded_cpu_masked_instanced": (None, [I, P, P, P, P, P, P, P, P, P, I]),
}


def lib_path() -> str:
    return _build.lib_path()


def load() -> C.CDLL:
    """Loads libimbart.so (built in-tree). Raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        raise ImbartError(f"libimbart is not built ({path} missing); run imbatracer_b200.build.build()")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        lib = load()
        msg = lib.imbart_last_error_string().decode(errors="replace")
        raise ImbartError(f"{what}: error {rc}: {msg}")


def last_error() -> tuple[int, str]:
    lib = load()
    return lib.imbart_last_error(), lib.imbart_last_error_string().decode(errors="replace")


def ptr(a) -> int | None:
    """Address of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data
    return a.data_ptr()
