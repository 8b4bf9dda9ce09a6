"""Scene input, ray files and image output over the C-ABI (host side, no GPU needed).

Reads the reference's scene.cfg / OBJ / camera.cfg / light.cfg files
(src/Application/SceneConfigurationReader.cpp, WFObjectReader.cpp, CameraManager.cpp,
LightSourceLoader.cpp), its headerless .rays files (6 float32 per ray,
SimpleRayTraverser.h:200-261), and writes hits files and PNG / PFM images
(ImagePNG.cpp:160-215).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import HRError, SceneInfo

IMAGE_PNG, IMAGE_PFM = 0, 1


def _chk(st: int, what: str):
    if st != 0:
        m = _lib.load().hr_io_last_error()
        raise HRError(st, f"{what}: {m.decode() if m else ''}")


@dataclass
class QuadLight:
    position: np.ndarray
    edge1: np.ndarray
    edge2: np.ndarray
    normal: np.ndarray
    intensity: np.ndarray


@dataclass
class Scene:
    """Key frames (K, V, 3) float32, triangles (N, 3) uint32, camera, lights, frame step, and
    the OBJ's shading normals and materials when it has them."""
    keyframes: np.ndarray
    faces: np.ndarray
    frame_step: float = 0.0
    camera: Optional[dict] = None
    lights: List[QuadLight] = field(default_factory=list)
    normals: Optional[np.ndarray] = None          # (M, 3) float32 shading normals
    normal_idx: Optional[np.ndarray] = None       # (N, 3) uint32, with normals
    albedo: Optional[np.ndarray] = None           # (K,) float32 material table
    materials: Optional[np.ndarray] = None        # (N,) uint32 material per triangle, with albedo


def _load(fn, path: str, threads: int) -> Scene:
    L = _lib.load()
    h = C.c_void_p()
    _chk(fn(str(path).encode(), threads, C.byref(h)), f"load {path}")
    try:
        info = SceneInfo()
        _chk(L.hr_scene_get_info(h, C.byref(info)), "scene info")
        k, v, n = info.num_keyframes, info.num_vertices, info.num_triangles
        kf = np.ctypeslib.as_array((C.c_float * (k * v * 3)).from_address(L.hr_scene_keyframes(h))).reshape(k, v, 3).copy()
        fa = np.ctypeslib.as_array((C.c_uint32 * (n * 3)).from_address(L.hr_scene_indices(h))).reshape(n, 3).copy()
        cam = None
        if info.has_camera:
            cam = dict(position=np.array(info.cam_position, np.float32), orientation=np.array(info.cam_orientation, np.float32),
                       up=np.array(info.cam_up, np.float32), fov=float(info.cam_fov_deg), res_x=int(info.width),
                       res_y=int(info.height))
        lights = []
        for i in range(info.num_lights):
            a = [(C.c_float * 3)() for _ in range(5)]
            _chk(L.hr_scene_get_light(h, i, *a), "light")
            lights.append(QuadLight(*[np.array(x, np.float32) for x in a]))
        nrm = nid = alb = mat = None
        if info.num_normals and n:
            nrm = np.ctypeslib.as_array((C.c_float * (3 * info.num_normals)).from_address(L.hr_scene_normals(h)))
            nrm = nrm.reshape(-1, 3).copy()
            nid = np.ctypeslib.as_array((C.c_uint32 * (n * 3)).from_address(L.hr_scene_normal_indices(h)))
            nid = nid.reshape(n, 3).copy()
        if info.num_materials and n:
            alb = np.ctypeslib.as_array((C.c_float * info.num_materials).from_address(L.hr_scene_material_albedo(h))).copy()
            mat = np.ctypeslib.as_array((C.c_uint32 * n).from_address(L.hr_scene_triangle_materials(h))).copy()
        return Scene(kf, fa, float(info.frame_step), cam, lights, nrm, nid, alb, mat)
    finally:
        L.hr_scene_free(h)


def load_scene(cfg_path: str, threads: int = 0) -> Scene:
    """A scene.cfg: static OBJ(s) or a key-frame sequence, with its camera and lights."""
    return _load(_lib.load().hr_scene_load, cfg_path, threads)


def load_obj(path: str, threads: int = 0) -> Scene:
    """One OBJ file as a one-key-frame scene (parsed in parallel over line chunks)."""
    return _load(_lib.load().hr_scene_load_obj, path, threads)


def read_rays(path: str):
    """(origins (n, 3), directions (n, 3)) float32 from a .rays file."""
    L = _lib.load()
    n = C.c_uint32()
    _chk(L.hr_rays_file_count(str(path).encode(), C.byref(n)), f"read {path}")
    buf = np.empty((n.value, 6), np.float32)
    _chk(L.hr_rays_file_read(str(path).encode(), buf.ctypes.data, n.value), f"read {path}")
    return np.ascontiguousarray(buf[:, :3]), np.ascontiguousarray(buf[:, 3:])


def write_rays(path: str, org, dirs):
    o = np.ascontiguousarray(org, np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    _chk(_lib.load().hr_rays_file_write(str(path).encode(), o.ctypes.data, d.ctypes.data, o.shape[0]), f"write {path}")


def write_hits(path: str, hid, t, u, v):
    a = [np.ascontiguousarray(hid, np.int32)] + [np.ascontiguousarray(x, np.float32) for x in (t, u, v)]
    _chk(_lib.load().hr_hits_file_write(str(path).encode(), *[x.ctypes.data for x in a], a[0].shape[0]),
         f"write {path}")


def write_image(path: str, rgb, width: int, height: int, fmt: int = IMAGE_PNG):
    a = np.ascontiguousarray(rgb, np.float32).reshape(-1)
    if a.size != width * height * 3:
        raise HRError(1, "write_image: rgb must hold 3 floats per pixel")
    _chk(_lib.load().hr_image_write(str(path).encode(), a.ctypes.data, width, height, fmt), f"write {path}")
