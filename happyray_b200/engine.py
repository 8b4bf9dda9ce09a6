"""Host-side engine over the C-ABI: the RTEngine interface of the reference.

Mirrors src/RT/RTEngine.h:36-68 (init, upload, buildAccStruct, setCamera, setLights,
renderFrame, setGridDensities, cleanup, getBoundingBoxDiagonalLength) with the same
argument meaning, plus the lower-level calls the tests and the bench need (ray queries,
grid download, device-pointer variants).  All numerical work happens in
libhappyray_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import GRID_TWO_LEVEL, GRID_UNIFORM, HRError, check  # noqa: F401


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):   # torch tensor on the context's device
        return a.data_ptr()
    if isinstance(a, int):
        return a
    raise TypeError(f"unsupported buffer type {type(a)}")


def _f3(x):
    return (C.c_float * 3)(*[float(v) for v in x])


class Engine:
    """One GPU context (hr_ctx).  `stream` is a cudaStream_t handle (int) or None."""

    def __init__(self, device: int = 0, stream: Optional[int] = None, lib=None):
        self.L = lib or _lib.load()
        ctx = C.c_void_p()
        st = self.L.hr_create(C.byref(ctx), device, C.c_void_p(stream) if stream else None)
        if st != 0:
            raise HRError(st, f"hr_create(device={device}) failed")
        self.ctx = ctx
        self.device = device
        self.res = (0, 0)
        self._keep = []

    # -- RTEngine::init / cleanup ------------------------------------------------
    @classmethod
    def init(cls, device: int = 0, stream: Optional[int] = None) -> "Engine":
        return cls(device, stream)

    def cleanup(self):
        if getattr(self, "ctx", None):
            self.L.hr_destroy(self.ctx)
            self.ctx = None

    close = cleanup

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.cleanup()

    def _chk(self, st, what):
        check(self.ctx, st, what, self.L)

    # -- RTEngine::upload(frame1, frame2, coeff) ---------------------------------
    def upload(self, frame1_xyz, frame2_xyz, tri_idx, coeff: float = 1.0):
        f1 = np.ascontiguousarray(frame1_xyz, np.float32).reshape(-1, 3)
        f2 = np.ascontiguousarray(frame2_xyz, np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(tri_idx, np.uint32).reshape(-1, 3)
        if f1.shape != f2.shape:
            raise HRError(1, "upload: key frames differ in vertex count")
        self._chk(self.L.hr_upload(self.ctx, _ptr(f1), _ptr(f2), f1.shape[0], _ptr(idx), idx.shape[0], coeff),
                  "hr_upload")

    def set_keyframes(self, frames_xyz, tri_idx):
        fr = np.ascontiguousarray(frames_xyz, np.float32)
        k, nv = fr.shape[0], fr.shape[1]
        idx = np.ascontiguousarray(tri_idx, np.uint32).reshape(-1, 3)
        self._chk(self.L.hr_set_keyframes(self.ctx, _ptr(fr), k, nv, _ptr(idx), idx.shape[0]), "hr_set_keyframes")

    def set_frame_time(self, t: float, step: float = 0.0):
        self._chk(self.L.hr_set_frame_time(self.ctx, t, step), "hr_set_frame_time")

    # -- RTEngine::setGridDensities / buildAccStruct -----------------------------
    def upload_scene(self, path: str, threads: int = 0):
        """Load a scene.cfg (or one .obj) and make it current: key frames, camera, lights,
        the OBJ's shading normals and materials (hr_scene_load / hr_scene_upload;
        CUDAApplication.cu:63-71 reads the same files at start-up).  Returns the camera
        resolution, or None without a camera."""
        h = C.c_void_p()
        fn = self.L.hr_scene_load_obj if str(path).lower().endswith(".obj") else self.L.hr_scene_load
        st = fn(str(path).encode(), threads, C.byref(h))
        if st != 0:
            m = self.L.hr_io_last_error()
            raise HRError(st, f"load {path}: {m.decode() if m else ''}")
        try:
            self._chk(self.L.hr_scene_upload(self.ctx, h), "hr_scene_upload")
            info = _lib.SceneInfo()
            self.L.hr_scene_get_info(h, C.byref(info))
            if info.has_camera and info.width > 0 and info.height > 0:
                self.res = (info.width, info.height)
                return self.res
            return None
        finally:
            self.L.hr_scene_free(h)

    def setGridDensities(self, top: float, leaf: float):
        self._chk(self.L.hr_set_grid_densities(self.ctx, top, leaf), "hr_set_grid_densities")

    def set_uniform_density(self, d: float):
        self._chk(self.L.hr_set_uniform_density(self.ctx, d), "hr_set_uniform_density")

    def buildAccStruct(self, kind: int = GRID_TWO_LEVEL, exact: bool = True):
        self._chk(self.L.hr_build(self.ctx, kind, int(exact)), "hr_build")

    build = buildAccStruct

    def grid_info(self) -> dict:
        gi = _lib.GridInfo()
        self._chk(self.L.hr_grid_get_info(self.ctx, C.byref(gi)), "hr_grid_get_info")
        return {"kind": gi.kind, "res": tuple(gi.res), "bounds_min": np.array(gi.bounds_min, np.float32),
                "bounds_max": np.array(gi.bounds_max, np.float32), "cell_size": np.array(gi.cell_size, np.float32),
                "cell_size_rcp": np.array(gi.cell_size_rcp, np.float32), "num_cells": gi.num_cells,
                "num_leaves": gi.num_leaves, "num_pairs": gi.num_pairs, "num_top_pairs": gi.num_top_pairs}

    def grid_download(self):
        gi = self.grid_info()
        cells = np.empty((gi["num_cells"], 2), np.uint32)
        leaves = np.empty((gi["num_leaves"], 2), np.uint32) if gi["kind"] == GRID_TWO_LEVEL else None
        prims = np.empty(gi["num_pairs"], np.uint32)
        self._chk(self.L.hr_grid_download(self.ctx, _ptr(cells), _ptr(leaves), _ptr(prims)), "hr_grid_download")
        return gi, cells, leaves, prims

    def vertices(self, nv: int):
        out = np.empty((nv, 4), np.float32)
        self._chk(self.L.hr_download_vertices(self.ctx, _ptr(out)), "hr_download_vertices")
        return out

    def set_timing(self, on: bool = True):
        self._chk(self.L.hr_set_timing(self.ctx, int(on)), "hr_set_timing")

    def stage_times(self):
        buf = (C.c_float * 16)()
        n = self.L.hr_get_stage_times(self.ctx, buf, 16)
        return [float(buf[i]) for i in range(n)]

    # -- RTEngine::setCamera / setLights ----------------------------------------
    def setCamera(self, position, orientation, up, fov: float, res_x: int, res_y: int):
        self._chk(self.L.hr_set_camera(self.ctx, _f3(position), _f3(orientation), _f3(up), fov, res_x, res_y),
                  "hr_set_camera")
        self.res = (res_x, res_y)

    def setLights(self, corner, edge1, edge2, emission, normals=None):
        """One light (corner, edge1, edge2: xyz; emission: float), or a collection: arrays of
        shape (n, 3) and n emissions, optional (n, 3) unit normals (RTEngine::setLights)."""
        c = np.asarray(corner, np.float32)
        if c.ndim == 1 and normals is None:
            self._chk(self.L.hr_set_light(self.ctx, _f3(corner), _f3(edge1), _f3(edge2), float(emission)),
                      "hr_set_light")
            return
        c = np.ascontiguousarray(c.reshape(-1, 3))
        e1 = np.ascontiguousarray(np.asarray(edge1, np.float32).reshape(-1, 3))
        e2 = np.ascontiguousarray(np.asarray(edge2, np.float32).reshape(-1, 3))
        em = np.ascontiguousarray(np.asarray(emission, np.float32).reshape(-1))
        nr = None if normals is None else np.ascontiguousarray(np.asarray(normals, np.float32).reshape(-1, 3))
        self._chk(self.L.hr_set_lights(self.ctx, c.shape[0], _ptr(c), _ptr(e1), _ptr(e2), _ptr(nr), _ptr(em)),
                  "hr_set_lights")

    def set_normals(self, normals_xyz=None, tri_normal_idx=None):
        """Shading normals for the path tracer (None removes them)."""
        if normals_xyz is None:
            self._chk(self.L.hr_set_normals(self.ctx, None, 0, None), "hr_set_normals")
            return
        n = np.ascontiguousarray(normals_xyz, np.float32).reshape(-1, 3)
        ix = np.ascontiguousarray(tri_normal_idx, np.uint32).reshape(-1, 3)
        self._chk(self.L.hr_set_normals(self.ctx, _ptr(n), n.shape[0], _ptr(ix)), "hr_set_normals")

    def set_materials(self, albedo=None, tri_material=None):
        """Per-triangle diffuse albedo table and indices for the path tracer (None removes them)."""
        if albedo is None:
            self._chk(self.L.hr_set_materials(self.ctx, None, 0, None), "hr_set_materials")
            return
        a = np.ascontiguousarray(albedo, np.float32).reshape(-1)
        ix = np.ascontiguousarray(tri_material, np.uint32).reshape(-1)
        self._chk(self.L.hr_set_materials(self.ctx, _ptr(a), a.shape[0], _ptr(ix)), "hr_set_materials")

    def set_integrator(self, ao_samples=8, ao_radius=-0.1, pt_bounces=4, albedo=0.7, seed=0x853c49e6748fea9b):
        self._chk(self.L.hr_set_integrator(self.ctx, ao_samples, ao_radius, pt_bounces, albedo, seed),
                  "hr_set_integrator")

    # -- RTEngine::renderFrame ---------------------------------------------------
    def renderFrame(self, framebuffer: Optional[np.ndarray], image_id: int, mode: int) -> np.ndarray:
        w, h = self.res
        fb = np.zeros((h * w, 3), np.float32) if framebuffer is None else framebuffer
        if fb.dtype != np.float32 or not fb.flags.c_contiguous or fb.size != w * h * 3:
            raise HRError(1, "renderFrame: frame buffer must be contiguous float32 with 3 floats per pixel")
        self._chk(self.L.hr_render(self.ctx, mode, image_id, _ptr(fb)), "hr_render")
        return fb

    def render_device(self, d_fb, image_id: int, mode: int):
        self._chk(self.L.hr_render_device(self.ctx, mode, image_id, _ptr(d_fb)), "hr_render_device")

    # -- ray queries ---------------------------------------------------------------
    def trace_rays(self, org, dirs):
        org = np.ascontiguousarray(org, np.float32).reshape(-1, 3)
        dirs = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        n = org.shape[0]
        hid = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        u = np.empty(n, np.float32)
        v = np.empty(n, np.float32)
        self._chk(self.L.hr_trace_rays(self.ctx, _ptr(org), _ptr(dirs), n, _ptr(hid), _ptr(t), _ptr(u), _ptr(v)),
                  "hr_trace_rays")
        return hid, t, u, v

    def trace_rays_file(self, rays_path: str, hits_path: str) -> int:
        """Ray query from a .rays file (6 float32 per ray, SimpleRayTraverser.h:200-261) to a
        hits file (int32 id, float32 t, u, v per ray).  Returns the number of rays."""
        from . import sceneio
        org, d = sceneio.read_rays(rays_path)
        hid, t, u, v = self.trace_rays(org, d)
        sceneio.write_hits(hits_path, hid, t, u, v)
        return org.shape[0]

    def trace_rays_device(self, d_org, d_dir, n, d_id, d_t, d_u, d_v):
        self._chk(self.L.hr_trace_rays_device(self.ctx, _ptr(d_org), _ptr(d_dir), n, _ptr(d_id), _ptr(d_t),
                                              _ptr(d_u), _ptr(d_v)), "hr_trace_rays_device")

    def trace_primary_device(self, d_id, d_t, d_u, d_v, d_stats=None):
        self._chk(self.L.hr_trace_primary_device(self.ctx, _ptr(d_id), _ptr(d_t), _ptr(d_u), _ptr(d_v),
                                                 _ptr(d_stats)), "hr_trace_primary_device")

    def render_rays_device(self, d_org, d_dir, n, image_id, d_fb):
        """Ray-file form of renderFrame mode 0: ray i shaded into pixel i (device buffers)."""
        self._chk(self.L.hr_render_rays_device(self.ctx, _ptr(d_org), _ptr(d_dir), n, image_id, _ptr(d_fb)),
                  "hr_render_rays_device")

    def occluded_device(self, d_org, d_dir, d_tmax, n, d_occ):
        self._chk(self.L.hr_occluded_device(self.ctx, _ptr(d_org), _ptr(d_dir), _ptr(d_tmax), n, _ptr(d_occ)),
                  "hr_occluded_device")

    def ray_count(self, reset: bool = False) -> int:
        n = C.c_uint64()
        self._chk(self.L.hr_get_ray_count(self.ctx, C.byref(n), int(reset)), "hr_get_ray_count")
        return int(n.value)

    def set_stats(self, on: bool = True):
        self._chk(self.L.hr_set_stats(self.ctx, int(on)), "hr_set_stats")

    def counters(self, reset: bool = False) -> dict:
        w = (C.c_uint64 * 8)()
        self._chk(self.L.hr_get_counters(self.ctx, w, int(reset)), "hr_get_counters")
        return {"rays": int(w[0]), "cells": int(w[1]), "tests": int(w[2]), "launches": int(w[3]),
                "rays2": int(w[4]), "cells2": int(w[5]), "tests2": int(w[6])}

    def render_times(self):
        buf = (C.c_float * 8)()
        n = self.L.hr_get_render_times(self.ctx, buf, 8)
        return [float(buf[i]) for i in range(n)]

    def sync(self):
        self._chk(self.L.hr_sync(self.ctx), "hr_sync")

    def getBoundingBoxDiagonalLength(self) -> float:
        return float(self.L.hr_bounds_diagonal(self.ctx))

    # -- build primitives ----------------------------------------------------------
    def exclusive_scan_device(self, d_data, n: int):
        self._chk(self.L.hr_exclusive_scan_device(self.ctx, _ptr(d_data), n), "hr_exclusive_scan_device")

    def radix_sort_pairs_device(self, d_keys, d_vals, n: int, key_bits: int):
        self._chk(self.L.hr_radix_sort_pairs_device(self.ctx, _ptr(d_keys), _ptr(d_vals), n, key_bits),
                  "hr_radix_sort_pairs_device")
