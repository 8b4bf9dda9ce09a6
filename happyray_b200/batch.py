"""Batched scenes over the C-ABI (hr_batch_* in include/happyray.h).

Many independent scenes are built as one segmented two-level-grid pipeline and rendered
by one persistent traversal launch, captured in a CUDA graph.  The reference has no
batched form: its RTEngine holds one scene (src/RT/RTEngine.cu:91-181), so the per-scene
Engine is the comparison path, and every scene's grid and image from a Batch are
bit-identical to what Engine gives for that scene.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import BatchScene, BatchTuning, GridInfo, HRError

ALL_SCENES = 0xFFFFFFFF


@dataclass
class SceneSpec:
    """One scene of a batch: mesh, pinhole camera (RTEngine::setCamera arguments) and
    integrator (ao_samples = 0: primary shading; > 0: AO with that many samples)."""
    vertices: np.ndarray            # (V, 3) float32
    faces: np.ndarray               # (N, 3) uint32, scene-local
    position: Sequence[float]
    orientation: Sequence[float]
    up: Sequence[float]
    fov: float
    width: int
    height: int
    ao_samples: int = 4
    top_density: float = 0.0        # <= 0: batch default 1/16
    leaf_density: float = 0.0       # <= 0: batch default 2


class Batch:
    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self.L = _lib.load()
        b = C.c_void_p()
        st = self.L.hr_batch_create(C.byref(b), device, C.c_void_p(stream) if stream else None)
        if st != 0:
            raise HRError(st, f"hr_batch_create(device={device}) failed")
        self.b = b
        self.device = device
        self.scenes: list[SceneSpec] = []
        self._keep = []

    def close(self):
        if getattr(self, "b", None):
            self.L.hr_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, st, what):
        if st != 0:
            m = self.L.hr_batch_last_error(self.b)
            raise HRError(st, f"{what}: {m.decode() if m else ''}")

    def set_scenes(self, scenes: Sequence[SceneSpec]):
        arr = (BatchScene * len(scenes))()
        keep = []
        for i, s in enumerate(scenes):
            v = np.ascontiguousarray(s.vertices, np.float32).reshape(-1, 3)
            f = np.ascontiguousarray(s.faces, np.uint32).reshape(-1, 3)
            keep += [v, f]
            r = arr[i]
            r.vertices_xyz = v.ctypes.data
            r.num_vertices = v.shape[0]
            r.indices = f.ctypes.data
            r.num_triangles = f.shape[0]
            r.cam_position[:] = [float(x) for x in s.position]
            r.cam_orientation[:] = [float(x) for x in s.orientation]
            r.cam_up[:] = [float(x) for x in s.up]
            r.cam_fov_deg = float(s.fov)
            r.width, r.height = int(s.width), int(s.height)
            r.ao_samples = int(s.ao_samples)
            r.top_density, r.leaf_density = float(s.top_density), float(s.leaf_density)
        self._chk(self.L.hr_batch_set_scenes(self.b, arr, len(scenes)), "set_scenes")
        self.scenes = list(scenes)

    def set_densities(self, top: float, leaf: float, scene: int = ALL_SCENES):
        self._chk(self.L.hr_batch_set_densities(self.b, scene, top, leaf), "set_densities")

    def set_launch(self, block_threads: int, tile_width: int):
        self._chk(self.L.hr_batch_set_launch(self.b, block_threads, tile_width), "set_launch")

    def set_integrator(self, ao_radius_fraction: float = 0.1, seed: int = 0x853c49e6748fea9b):
        self._chk(self.L.hr_batch_set_integrator(self.b, ao_radius_fraction, seed), "set_integrator")

    def set_graph(self, use_graph: bool):
        self._chk(self.L.hr_batch_set_graph(self.b, 1 if use_graph else 0), "set_graph")

    def set_vertices(self, xyz: np.ndarray):
        """New positions for all scenes' vertices (scenes concatenated, same meshes)."""
        a = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        self._chk(self.L.hr_batch_set_vertices(self.b, a.ctypes.data, a.shape[0]), "set_vertices")

    def run(self, image_id: int = 0):
        """One step: rebuild every grid and render every scene (synchronous)."""
        self._chk(self.L.hr_batch_run(self.b, image_id), "run")

    def times(self):
        """(build ms, render ms, total ms) of the last step."""
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        self._chk(self.L.hr_batch_get_times(self.b, C.byref(a), C.byref(b), C.byref(c)), "times")
        return a.value, b.value, c.value

    def counters(self, reset: bool = False):
        """[rays, kernels launched, scenes, pixels, secondary rays, 0, 0, 0]"""
        out = (C.c_uint64 * 8)()
        self._chk(self.L.hr_batch_get_counters(self.b, out, 1 if reset else 0), "counters")
        return list(out)

    def image(self, scene: int) -> np.ndarray:
        s = self.scenes[scene]
        out = np.empty((s.height, s.width, 3), np.float32)
        self._chk(self.L.hr_batch_get_image(self.b, scene, out.ctypes.data), "image")
        return out

    def download_images(self, out: np.ndarray) -> np.ndarray:
        """All framebuffers, scenes concatenated (float32, 3 per pixel) into `out`."""
        if out.dtype != np.float32 or not out.flags.c_contiguous:
            raise HRError(1, "download_images: out must be contiguous float32")
        self._chk(self.L.hr_batch_download_images(self.b, out.ctypes.data, out.size), "download_images")
        return out

    def image_device(self, scene: int) -> int:
        p = C.c_void_p()
        self._chk(self.L.hr_batch_image_device(self.b, scene, C.byref(p)), "image_device")
        return p.value

    def grid_info(self, scene: int) -> dict:
        gi = GridInfo()
        self._chk(self.L.hr_batch_grid_info(self.b, scene, C.byref(gi)), "grid_info")
        return {"kind": gi.kind, "res": tuple(gi.res), "bounds_min": tuple(gi.bounds_min),
                "bounds_max": tuple(gi.bounds_max), "cell_size": tuple(gi.cell_size),
                "cell_size_rcp": tuple(gi.cell_size_rcp), "num_cells": gi.num_cells, "num_leaves": gi.num_leaves,
                "num_pairs": gi.num_pairs, "num_top_pairs": gi.num_top_pairs}

    def grid_download(self, scene: int):
        """(top cells uint32[C, 2], leaves uint32[L, 2], primitives uint32[P]) of one scene,
        in the per-scene layout of Engine.grid_download."""
        gi = self.grid_info(scene)
        cells = np.zeros((gi["num_cells"], 2), np.uint32)
        leaves = np.zeros((gi["num_leaves"], 2), np.uint32)
        prims = np.zeros(gi["num_pairs"], np.uint32)
        self._chk(self.L.hr_batch_grid_download(self.b, scene, cells.ctypes.data, leaves.ctypes.data,
                                                prims.ctypes.data), "grid_download")
        return cells, leaves, prims

    def autotune(self, reps: int = 3) -> dict:
        t = BatchTuning()
        self._chk(self.L.hr_batch_autotune(self.b, reps, C.byref(t)), "autotune")
        return {"top_density": t.top_density, "leaf_density": t.leaf_density, "block_threads": t.block_threads,
                "tile_width": t.tile_width, "ms_per_step": t.ms_per_step, "trials": t.trials}
