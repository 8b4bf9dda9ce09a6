"""Instanced two-level grid hierarchy (hr_hier_* in include/happyray.h).

Mirrors the reference's TLGRIDHIERARCHY engine configuration (RTEngine.cu:68-73;
TwoLevelGridHierarchy.h, TLGridHierarchySortBuilder.cu, TLGridHierarchyTraverser.h):
objects are consecutive triangle ranges of one mesh in their own coordinates, each with
its own uniform grid; instances (object, world -> object map, world box) are binned into
a uniform grid over their boxes.  A rigid-body frame changes the instances only, and
build() then rebuilds the instance grid alone.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import HRError

# one hr_instance: object index, the three world -> object rows, world box
INSTANCE_DTYPE = np.dtype([("obj", "<u4"), ("m", "<f4", 12), ("bmin", "<f4", 3), ("bmax", "<f4", 3)])
OBJECT_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("cs", "<f4", 3), ("rcp", "<f4", 3),
                         ("res", "<i4", 3), ("cell_off", "<u4"), ("tri_begin", "<u4"), ("tri_count", "<u4")])


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Hierarchy:
    def __init__(self, device: int = 0, stream=None):
        self._lib = L.load()
        self._h = C.c_void_p()
        self._check(self._lib.hr_hier_create(C.byref(self._h), device, stream), "create")
        self._keep = []

    def _check(self, st, what):
        if st != L.HR_OK:
            msg = ""
            if self._h:
                m = self._lib.hr_hier_last_error(self._h)
                msg = m.decode() if m else ""
            raise HRError(st, f"{what}: {msg}")

    def close(self):
        if self._h:
            self._lib.hr_hier_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_objects(self, vertices, faces, object_tri_counts):
        v = np.ascontiguousarray(vertices, np.float32)
        f = np.ascontiguousarray(faces, np.uint32)
        c = np.ascontiguousarray(object_tri_counts, np.uint32)
        self._check(self._lib.hr_hier_set_objects(self._h, _p(v), v.shape[0], _p(f), f.shape[0], _p(c), c.shape[0]),
                    "set_objects")

    def set_instances(self, inst):
        a = np.ascontiguousarray(inst, INSTANCE_DTYPE)
        self._check(self._lib.hr_hier_set_instances(self._h, _p(a), a.shape[0]), "set_instances")

    def set_densities(self, top: float = 1.2, objects: float = 1.2):
        self._check(self._lib.hr_hier_set_densities(self._h, top, objects), "set_densities")

    def build(self):
        self._check(self._lib.hr_hier_build(self._h), "build")

    def info(self) -> dict:
        i = L.HierInfo()
        self._check(self._lib.hr_hier_get_info(self._h, C.byref(i)), "info")
        return {k: (list(getattr(i, k)) if k in ("top_res", "top_bmin", "top_bmax") else getattr(i, k))
                for k, _ in L.HierInfo._fields_}

    def download(self):
        """(objects, object cells (C, 2), triangle lists, instance-grid cells, instance lists)"""
        i = self.info()
        objs = np.empty(i["num_objects"], OBJECT_DTYPE)
        oc = np.empty((i["num_object_cells"], 2), np.uint32)
        tri = np.empty(i["num_pairs"], np.uint32)
        tc = np.empty((i["num_top_cells"], 2), np.uint32)
        ii = np.empty(i["num_top_pairs"], np.uint32)
        self._check(self._lib.hr_hier_download(self._h, _p(objs), _p(oc), _p(tri), _p(tc), _p(ii)), "download")
        return objs, oc, tri, tc, ii

    def trace_rays(self, org, dirs, out=None):
        """Closest hits: (instance id, triangle id, t, u, v), -1 ids on a miss.  out: five
        caller arrays of n elements (int32, int32, float32 x 3) to fill instead of new ones,
        e.g. page-locked ones, whose copies run at the full host link rate."""
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        n = org.shape[0]
        if out is None:
            out = [np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32),
                   np.empty(n, np.float32)]
        else:
            want = (np.int32, np.int32, np.float32, np.float32, np.float32)
            if len(out) != 5 or any(a.dtype != w or a.size != n or not a.flags.c_contiguous for a, w in zip(out, want)):
                raise ValueError("trace_rays: out must be five contiguous arrays of n int32, int32, float32 x 3")
        self._check(self._lib.hr_hier_trace_rays(self._h, _p(org), _p(dirs), n, *[_p(a) for a in out]), "trace_rays")
        return tuple(out)

    def trace_rays_device(self, org, dirs, inst, tri, t, u, v):
        """Device form (torch CUDA tensors: org/dirs (n, 3) float32; int32 and float32 outputs)."""
        n = org.shape[0]
        self._check(self._lib.hr_hier_trace_rays_device(self._h, org.data_ptr(), dirs.data_ptr(), n, inst.data_ptr(),
                                                        tri.data_ptr(), t.data_ptr(), u.data_ptr(), v.data_ptr()),
                    "trace_rays_device")

    def trace_stats_device(self, org, dirs, inst, tri, t, u, v, stats):
        """trace_rays_device plus 5 counters per ray in stats ((n, 5) int32 tensor): instance-grid
        cells, instance boxes tested, instances entered, object-grid cells, triangle tests."""
        n = org.shape[0]
        self._check(self._lib.hr_hier_trace_stats_device(self._h, org.data_ptr(), dirs.data_ptr(), n, inst.data_ptr(),
                                                         tri.data_ptr(), t.data_ptr(), u.data_ptr(), v.data_ptr(),
                                                         stats.data_ptr()), "trace_stats_device")

    def occluded(self, org, dirs, tmax):
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        n = org.shape[0]
        tm = np.ascontiguousarray(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        occ = np.empty(n, np.uint8)
        self._check(self._lib.hr_hier_occluded(self._h, _p(org), _p(dirs), _p(tm), n, _p(occ)), "occluded")
        return occ.astype(bool)


def read_instances(path: str) -> np.ndarray:
    """The reference's instances file (WFObjectReader.cpp:762-825)."""
    lib = L.load()
    n = C.c_uint32()
    st = lib.hr_instances_file_read(path.encode(), None, 0, C.byref(n))
    if st != L.HR_OK:
        raise HRError(st, lib.hr_io_last_error().decode())
    out = np.zeros(n.value, INSTANCE_DTYPE)
    st = lib.hr_instances_file_read(path.encode(), _p(out), n.value, C.byref(n))
    if st != L.HR_OK:
        raise HRError(st, lib.hr_io_last_error().decode())
    return out


def write_instances(path: str, inst):
    lib = L.load()
    a = np.ascontiguousarray(inst, INSTANCE_DTYPE)
    st = lib.hr_instances_file_write(path.encode(), _p(a), a.shape[0])
    if st != L.HR_OK:
        raise HRError(st, lib.hr_io_last_error().decode())
