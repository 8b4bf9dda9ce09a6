"""ctypes binding of libhappyray_b200.so (C-ABI in include/happyray.h).

The product path always runs the CUDA library: if the shared object is missing or
cannot be loaded, every call raises HRError -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

PKG = Path(__file__).resolve().parent
IEEE_LIB_PATH = PKG / "libhappyray_b200.so"
FAST_LIB_PATH = PKG / "libhappyray_b200_fast.so"
# HAPPYRAY_B200_ARITH=fast selects the fast-arithmetic build (results within the ray
# queries' floating-point tolerance instead of bit-exact); the default is the IEEE build
LIB_PATH = FAST_LIB_PATH if os.environ.get("HAPPYRAY_B200_ARITH", "").lower() == "fast" else IEEE_LIB_PATH

HR_OK = 0
STATUS = {0: "HR_OK", 1: "HR_ERR_INVALID_ARG", 2: "HR_ERR_OUT_OF_MEMORY", 3: "HR_ERR_CAPACITY_RETRY",
          4: "HR_ERR_DEVICE", 5: "HR_ERR_TIMEOUT", 6: "HR_ERR_NOT_READY"}

GRID_UNIFORM, GRID_TWO_LEVEL = 0, 1
RENDER_PRIMARY, RENDER_PATH, RENDER_PATH_SINGLE_KERNEL, RENDER_AO = 0, 1, 2, 3


class HRError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class GridInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("res", C.c_int32 * 3), ("bounds_min", C.c_float * 3),
                ("bounds_max", C.c_float * 3), ("cell_size", C.c_float * 3), ("cell_size_rcp", C.c_float * 3),
                ("num_cells", C.c_uint32), ("num_leaves", C.c_uint32), ("num_pairs", C.c_uint32),
                ("num_top_pairs", C.c_uint32)]


# every exported symbol with (restype, argtypes); the CPU tests check the .so exports them all
P = C.c_void_p
SIGNATURES = {
    "hr_create": (C.c_int, [C.POINTER(P), C.c_int32, P]),
    "hr_destroy": (None, [P]),
    "hr_last_error": (C.c_char_p, [P]),
    "hr_upload": (C.c_int, [P, P, P, C.c_uint32, P, C.c_uint32, C.c_float]),
    "hr_set_keyframes": (C.c_int, [P, P, C.c_uint32, C.c_uint32, P, C.c_uint32]),
    "hr_set_frame_time": (C.c_int, [P, C.c_float, C.c_float]),
    "hr_set_grid_densities": (C.c_int, [P, C.c_float, C.c_float]),
    "hr_set_uniform_density": (C.c_int, [P, C.c_float]),
    "hr_build": (C.c_int, [P, C.c_int32, C.c_int32]),
    "hr_grid_get_info": (C.c_int, [P, C.POINTER(GridInfo)]),
    "hr_grid_download": (C.c_int, [P, P, P, P]),
    "hr_set_timing": (C.c_int, [P, C.c_int32]),
    "hr_get_stage_times": (C.c_int32, [P, P, C.c_int32]),
    "hr_download_vertices": (C.c_int, [P, P]),
    "hr_set_camera": (C.c_int, [P, P, P, P, C.c_float, C.c_int32, C.c_int32]),
    "hr_set_light": (C.c_int, [P, P, P, P, C.c_float]),
    "hr_set_lights": (C.c_int, [P, C.c_uint32, P, P, P, P, P]),
    "hr_set_normals": (C.c_int, [P, P, C.c_uint32, P]),
    "hr_set_materials": (C.c_int, [P, P, C.c_uint32, P]),
    "hr_render_rays_device": (C.c_int, [P, P, P, C.c_uint32, C.c_int32, P]),
    "hr_set_integrator": (C.c_int, [P, C.c_int32, C.c_float, C.c_int32, C.c_float, C.c_uint64]),
    "hr_render": (C.c_int, [P, C.c_int32, C.c_int32, P]),
    "hr_render_device": (C.c_int, [P, C.c_int32, C.c_int32, P]),
    "hr_trace_rays": (C.c_int, [P, P, P, C.c_uint32, P, P, P, P]),
    "hr_trace_rays_device": (C.c_int, [P, P, P, C.c_uint32, P, P, P, P]),
    "hr_trace_primary_device": (C.c_int, [P, P, P, P, P, P]),
    "hr_occluded_device": (C.c_int, [P, P, P, P, C.c_uint32, P]),
    "hr_get_ray_count": (C.c_int, [P, C.POINTER(C.c_uint64), C.c_int32]),
    "hr_set_stats": (C.c_int, [P, C.c_int32]),
    "hr_get_counters": (C.c_int, [P, C.POINTER(C.c_uint64), C.c_int32]),
    "hr_get_render_times": (C.c_int32, [P, P, C.c_int32]),
    "hr_sync": (C.c_int, [P]),
    "hr_bounds_diagonal": (C.c_float, [P]),
    "hr_exclusive_scan_device": (C.c_int, [P, P, C.c_uint32]),
    "hr_radix_sort_pairs_device": (C.c_int, [P, P, P, C.c_uint32, C.c_int32]),
    "hr_radix_sort_pairs_noalloc": (C.c_int, [P, P, P, C.c_uint32, C.c_int32]),
    "hr_probe_l2_read": (C.c_int, [P, C.POINTER(C.c_double)]),
    # batched scenes
    "hr_batch_create": (C.c_int, [C.POINTER(P), C.c_int32, P]),
    "hr_batch_destroy": (None, [P]),
    "hr_batch_last_error": (C.c_char_p, [P]),
    "hr_batch_set_scenes": (C.c_int, [P, P, C.c_uint32]),
    "hr_batch_set_densities": (C.c_int, [P, C.c_uint32, C.c_float, C.c_float]),
    "hr_batch_set_launch": (C.c_int, [P, C.c_int32, C.c_int32]),
    "hr_batch_set_integrator": (C.c_int, [P, C.c_float, C.c_uint64]),
    "hr_batch_set_graph": (C.c_int, [P, C.c_int32]),
    "hr_batch_set_vertices": (C.c_int, [P, P, C.c_uint32]),
    "hr_batch_run": (C.c_int, [P, C.c_int32]),
    "hr_batch_get_times": (C.c_int, [P, P, P, P]),
    "hr_batch_get_counters": (C.c_int, [P, P, C.c_int32]),
    "hr_batch_get_image": (C.c_int, [P, C.c_uint32, P]),
    "hr_batch_image_device": (C.c_int, [P, C.c_uint32, P]),
    "hr_batch_download_images": (C.c_int, [P, P, C.c_uint64]),
    "hr_batch_grid_info": (C.c_int, [P, C.c_uint32, C.POINTER(GridInfo)]),
    "hr_batch_grid_download": (C.c_int, [P, C.c_uint32, P, P, P]),
    "hr_batch_autotune": (C.c_int, [P, C.c_int32, P]),
    # served rendering
    "hr_server_create": (C.c_int, [C.POINTER(P), C.c_int32, C.c_uint64, C.c_int32]),
    "hr_server_destroy": (None, [P]),
    "hr_server_last_error": (C.c_char_p, [P]),
    "hr_server_add_scene": (C.c_int, [P, P, C.c_uint32, C.c_uint32, P, C.c_uint32, C.c_float, C.c_float,
                                      C.POINTER(C.c_uint32)]),
    "hr_server_submit": (C.c_int, [P, P, C.POINTER(C.c_uint64)]),
    "hr_server_wait": (C.c_int, [P, C.c_uint64, C.c_int32]),
    "hr_server_drain": (C.c_int, [P, C.c_int32]),
    "hr_server_request_info": (C.c_int, [P, C.c_uint64, P]),
    "hr_server_get_stats": (C.c_int, [P, P]),
    "hr_server_set_watchdog": (C.c_int, [P, C.c_int32]),
    "hr_server_inject_stall": (C.c_int, [P, C.c_uint32, C.c_int32]),
    # scene input, ray files, images
    "hr_scene_load": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(P)]),
    "hr_scene_load_obj": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(P)]),
    "hr_scene_free": (None, [P]),
    "hr_io_last_error": (C.c_char_p, []),
    "hr_scene_get_info": (C.c_int, [P, P]),
    "hr_scene_keyframes": (P, [P]),
    "hr_scene_indices": (P, [P]),
    "hr_scene_normals": (P, [P]),
    "hr_scene_normal_indices": (P, [P]),
    "hr_scene_material_albedo": (P, [P]),
    "hr_scene_triangle_materials": (P, [P]),
    "hr_scene_get_light": (C.c_int, [P, C.c_uint32, P, P, P, P, P]),
    "hr_scene_upload": (C.c_int, [P, P]),
    "hr_rays_file_count": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32)]),
    "hr_rays_file_read": (C.c_int, [C.c_char_p, P, C.c_uint32]),
    "hr_rays_file_write": (C.c_int, [C.c_char_p, P, P, C.c_uint32]),
    "hr_hits_file_write": (C.c_int, [C.c_char_p, P, P, P, P, C.c_uint32]),
    "hr_image_write": (C.c_int, [C.c_char_p, P, C.c_int32, C.c_int32, C.c_int32]),
    # instanced two-level grid hierarchy
    "hr_hier_create": (C.c_int, [C.POINTER(P), C.c_int32, P]),
    "hr_hier_destroy": (None, [P]),
    "hr_hier_last_error": (C.c_char_p, [P]),
    "hr_hier_set_objects": (C.c_int, [P, P, C.c_uint32, P, C.c_uint32, P, C.c_uint32]),
    "hr_hier_set_instances": (C.c_int, [P, P, C.c_uint32]),
    "hr_hier_set_densities": (C.c_int, [P, C.c_float, C.c_float]),
    "hr_hier_build": (C.c_int, [P]),
    "hr_hier_get_info": (C.c_int, [P, P]),
    "hr_hier_download": (C.c_int, [P, P, P, P, P, P]),
    "hr_hier_trace_rays": (C.c_int, [P, P, P, C.c_uint32, P, P, P, P, P]),
    "hr_hier_trace_rays_device": (C.c_int, [P, P, P, C.c_uint32, P, P, P, P, P]),
    "hr_hier_trace_stats_device": (C.c_int, [P, P, P, C.c_uint32, P, P, P, P, P, P]),
    "hr_hier_occluded": (C.c_int, [P, P, P, P, C.c_uint32, P]),
    "hr_instances_file_read": (C.c_int, [C.c_char_p, P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "hr_instances_file_write": (C.c_int, [C.c_char_p, P, C.c_uint32]),
}


class Instance(C.Structure):
    """hr_instance"""
    _fields_ = [("object", C.c_uint32), ("m", C.c_float * 12), ("bmin", C.c_float * 3), ("bmax", C.c_float * 3)]


class HierInfo(C.Structure):
    """hr_hier_info"""
    _fields_ = [("num_objects", C.c_uint32), ("num_instances", C.c_uint32), ("num_triangles", C.c_uint32),
                ("num_object_cells", C.c_uint32), ("num_pairs", C.c_uint32), ("top_res", C.c_int32 * 3),
                ("num_top_cells", C.c_uint32), ("num_top_pairs", C.c_uint32), ("top_bmin", C.c_float * 3),
                ("top_bmax", C.c_float * 3), ("launches", C.c_uint64)]


class HierObject(C.Structure):
    """hr_hier_object"""
    _fields_ = [("bmin", C.c_float * 3), ("bmax", C.c_float * 3), ("cell_size", C.c_float * 3),
                ("cell_size_rcp", C.c_float * 3), ("res", C.c_int32 * 3), ("first_cell", C.c_uint32),
                ("first_triangle", C.c_uint32), ("num_triangles", C.c_uint32)]


class BatchScene(C.Structure):
    """hr_batch_scene"""
    _fields_ = [("vertices_xyz", P), ("num_vertices", C.c_uint32), ("indices", P), ("num_triangles", C.c_uint32),
                ("cam_position", C.c_float * 3), ("cam_orientation", C.c_float * 3), ("cam_up", C.c_float * 3),
                ("cam_fov_deg", C.c_float), ("width", C.c_int32), ("height", C.c_int32), ("ao_samples", C.c_int32),
                ("top_density", C.c_float), ("leaf_density", C.c_float)]


class BatchTuning(C.Structure):
    """hr_batch_tuning"""
    _fields_ = [("top_density", C.c_float), ("leaf_density", C.c_float), ("block_threads", C.c_int32),
                ("tile_width", C.c_int32), ("ms_per_step", C.c_float), ("trials", C.c_int32)]


class SceneInfo(C.Structure):
    """hr_scene_info"""
    _fields_ = [("num_vertices", C.c_uint32), ("num_triangles", C.c_uint32), ("num_keyframes", C.c_uint32),
                ("frame_step", C.c_float), ("has_camera", C.c_int32), ("cam_position", C.c_float * 3),
                ("cam_orientation", C.c_float * 3), ("cam_up", C.c_float * 3), ("cam_fov_deg", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32), ("num_lights", C.c_uint32),
                ("num_normals", C.c_uint32), ("num_materials", C.c_uint32)]


class Request(C.Structure):
    """hr_request"""
    _fields_ = [("scene", C.c_uint32), ("frame_time", C.c_float), ("kind", C.c_int32), ("mode", C.c_int32),
                ("spp", C.c_int32), ("cam_position", C.c_float * 3), ("cam_orientation", C.c_float * 3),
                ("cam_up", C.c_float * 3), ("cam_fov_deg", C.c_float), ("width", C.c_int32), ("height", C.c_int32),
                ("seed", C.c_uint64), ("out_rgb", P), ("ray_org", P), ("ray_dir", P), ("num_rays", C.c_uint32),
                ("out_id", P), ("out_t", P), ("out_u", P), ("out_v", P)]


class RequestInfo(C.Structure):
    """hr_request_info"""
    _fields_ = [("status", C.c_int32), ("wave", C.c_uint32), ("submit_ns", C.c_uint64), ("admit_ns", C.c_uint64),
                ("done_ns", C.c_uint64)]


class ServerStats(C.Structure):
    """hr_server_stats"""
    _fields_ = [("completed", C.c_uint64), ("failed", C.c_uint64), ("waves", C.c_uint64), ("rebuilds", C.c_uint64),
                ("rays", C.c_uint64), ("resident_bytes", C.c_uint64), ("peak_inflight_bytes", C.c_uint64),
                ("launches", C.c_uint64), ("trace_ms", C.c_double), ("watchdog_trips", C.c_uint64)]


_lock = threading.Lock()
_libs = {}


def load(path: Path | None = None):
    """Load a CUDA library: `path`, else the build HAPPYRAY_B200_ARITH selects (raises
    HRError if it is missing: no fallback).  Each library is loaded once, with its own
    symbols (RTLD_LOCAL), so the IEEE and the fast build can be used side by side."""
    p = Path(path).resolve() if path else LIB_PATH
    with _lock:
        if p in _libs:
            return _libs[p]
        if not p.exists():
            raise HRError(4, f"{p} is missing; build it with happyray_b200.build.build()")
        L = C.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _libs[p] = L
        return L


def load_fast():
    """The fast-arithmetic build (libhappyray_b200_fast.so)."""
    return load(FAST_LIB_PATH)


def check(ctx, status: int, what: str = "", lib=None):
    if status != HR_OK:
        msg = ""
        if ctx:
            m = (lib or load()).hr_last_error(ctx)
            msg = m.decode() if m else ""
        raise HRError(status, f"{what}: {msg}" if what else msg)
