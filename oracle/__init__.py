"""ctypes bindings of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's build and traversal
(javorkk/happyray, files cited in hr_oracle.c) on the CPU.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference arm import it, and only
as the checker.  The product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lock = threading.Lock()
_lib = None

UG, TL = 0, 1


class Grid(C.Structure):
    _fields_ = [("bmin", C.c_float * 3), ("bmax", C.c_float * 3), ("res", C.c_int32 * 3),
                ("cs", C.c_float * 3), ("rcp", C.c_float * 3), ("ncells", C.c_uint32)]


class Scene(C.Structure):
    _fields_ = [("v4", C.c_void_p), ("idx", C.c_void_p), ("ntri", C.c_uint32), ("kind", C.c_int32),
                ("g", Grid), ("cells", C.c_void_p), ("leaves", C.c_void_p), ("prims", C.c_void_p),
                ("nrm3", C.c_void_p), ("alb", C.c_void_p)]


class Obj(C.Structure):
    _fields_ = [("bmin", C.c_float * 3), ("bmax", C.c_float * 3), ("cs", C.c_float * 3), ("rcp", C.c_float * 3),
                ("res", C.c_int32 * 3), ("cell_off", C.c_uint32), ("tri_begin", C.c_uint32), ("tri_count", C.c_uint32)]


class Inst(C.Structure):
    _fields_ = [("obj", C.c_uint32), ("m", C.c_float * 12), ("bmin", C.c_float * 3), ("bmax", C.c_float * 3)]


class Hier(C.Structure):
    _fields_ = [("v4", C.c_void_p), ("idx", C.c_void_p), ("ntri", C.c_uint32), ("nobj", C.c_uint32),
                ("ninst", C.c_uint32), ("objs", C.c_void_p), ("inst", C.c_void_p), ("top", Grid),
                ("top_cells", C.c_void_p), ("inst_ids", C.c_void_p), ("obj_cells", C.c_void_p), ("prims", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("top_left", C.c_float * 3), ("step_x", C.c_float * 3),
                ("step_y", C.c_float * 3), ("w", C.c_int32), ("h", C.c_int32)]


class Light(C.Structure):
    _fields_ = [("corner", C.c_float * 3), ("e1", C.c_float * 3), ("e2", C.c_float * 3),
                ("normal", C.c_float * 3), ("emission", C.c_float)]


def build():
    """Compile liboracle.so from oracle/hr_oracle.c (make)."""
    src = HERE / "hr_oracle.c"
    if LIB.exists() and LIB.stat().st_mtime >= max(src.stat().st_mtime, (HERE / "hr_oracle.h").stat().st_mtime):
        return LIB
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(str(LIB))
            P = C.c_void_p
            F = C.c_float
            U32 = C.c_uint32
            I32 = C.c_int32
            U64 = C.c_uint64
            sig = {
                "orc_lerp_bounds": (None, [P, P, U32, F, P, P, P]),
                "orc_grid_setup": (None, [P, P, U32, F, C.POINTER(Grid)]),
                "orc_pow_third": (F, [F]),
                "orc_build_ug": (C.c_int, [P, P, U32, P, P, F, C.c_int, C.POINTER(Grid), C.POINTER(P), C.POINTER(P), C.POINTER(U32)]),
                "orc_build_tl": (C.c_int, [P, P, U32, P, P, F, F, C.POINTER(Grid), C.POINTER(P), C.POINTER(P), C.POINTER(U32),
                                           C.POINTER(P), C.POINTER(U32), C.POINTER(U32)]),
                "orc_free": (None, [P]),
                "orc_camera_init": (None, [C.POINTER(Camera), P, P, P, F, I32, I32]),
                "orc_primary_rays": (None, [C.POINTER(Camera), P, P]),
                "orc_trace": (None, [C.POINTER(Scene), P, P, U32, P, P, P, P, P]),
                "orc_trace_primary": (None, [C.POINTER(Scene), C.POINTER(Camera), P, P, P, P, P]),
                "orc_occluded": (None, [C.POINTER(Scene), P, P, P, U32, P]),
                "orc_render_ao": (None, [C.POINTER(Scene), C.POINTER(Camera), I32, F, U64, I32, P, U32, P]),
                "orc_render_primary": (None, [C.POINTER(Scene), C.POINTER(Camera), I32, U64, P]),
                "orc_log_series": (F, [F]),
                "orc_render_rays": (None, [C.POINTER(Scene), P, P, U32, I32, P]),
                "orc_render_pt": (None, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(Light), I32, I32, F, F, U64, I32, P, U32, P]),
                "orc_brute_f64": (None, [P, P, U32, P, P, U32, P, P, P, P, P]),
                "orc_sincos2pi": (None, [F, C.POINTER(F), C.POINTER(F)]),
                "orc_pcg32_first_floats": (F, [U64, U64, I32, P]),
                "orc_num_threads": (C.c_int, []),
                "orc_hier_build": (C.c_int, [P, P, U32, P, U32, P, U32, F, F, P, C.POINTER(Grid), C.POINTER(P),
                                             C.POINTER(U32), C.POINTER(P), C.POINTER(U32), C.POINTER(P), C.POINTER(P),
                                             C.POINTER(U32)]),
                "orc_hier_trace": (None, [C.POINTER(Hier), P, P, P, U32, C.c_int, P, P, P, P, P]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f3(x):
    return (C.c_float * 3)(*[float(v) for v in x])


def num_threads() -> int:
    return int(lib().orc_num_threads())


def lerp_bounds(f1: np.ndarray, f2: np.ndarray, coeff: float):
    """Keyframe interpolation + padded bounds (WFObjectUploader.h:82-114)."""
    f1 = np.ascontiguousarray(f1, np.float32)
    f2 = np.ascontiguousarray(f2, np.float32)
    nv = f1.shape[0]
    out = np.empty((nv, 4), np.float32)
    bmin = np.empty(3, np.float32)
    bmax = np.empty(3, np.float32)
    lib().orc_lerp_bounds(_p(f1), _p(f2), nv, coeff, _p(out), _p(bmin), _p(bmax))
    return out, bmin, bmax


def pow_third(x: float) -> float:
    return float(lib().orc_pow_third(x))


class Built:
    """Result of an oracle build; keeps the arrays alive for traversal calls."""

    def __init__(self, kind, v4, idx, grid, cells, leaves, prims, npairs, ntop_pairs=0):
        self.kind = kind
        self.v4 = v4
        self.idx = idx
        self.grid = grid
        self.cells = cells
        self.leaves = leaves
        self.prims = prims
        self.npairs = npairs
        self.ntop_pairs = ntop_pairs

    @property
    def res(self):
        return tuple(int(r) for r in self.grid.res)

    def scene(self) -> Scene:
        s = Scene()
        s.v4 = _p(self.v4)
        s.idx = _p(self.idx)
        s.ntri = self.idx.shape[0]
        s.kind = self.kind
        s.g = self.grid
        s.cells = _p(self.cells)
        s.leaves = _p(self.leaves) if self.leaves is not None else None
        s.prims = _p(self.prims)
        nrm3 = getattr(self, "nrm3", None)
        alb = getattr(self, "alb", None)
        s.nrm3 = _p(nrm3) if nrm3 is not None else None
        s.alb = _p(alb) if alb is not None else None
        self._scene = s
        return s

    def set_shading(self, normals_xyz=None, tri_normal_idx=None, albedo=None, tri_material=None):
        """Path-tracer shading normals (gathered to 3 per triangle) and per-triangle albedo."""
        self.nrm3 = None if normals_xyz is None else np.ascontiguousarray(
            np.asarray(normals_xyz, np.float32).reshape(-1, 3)[np.asarray(tri_normal_idx).reshape(-1, 3)])
        self.alb = None if albedo is None else np.ascontiguousarray(
            np.asarray(albedo, np.float32)[np.asarray(tri_material).reshape(-1)])

    def diag(self) -> np.float32:
        d = np.array(self.grid.bmax, np.float32) - np.array(self.grid.bmin, np.float32)
        return np.float32(np.sqrt(np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])))


def _take(ptr, n, dtype=np.uint32):
    if n == 0:
        lib().orc_free(ptr)
        return np.zeros(0, dtype)
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint32)), shape=(n,)).copy()
    lib().orc_free(ptr)
    return arr


def build_ug(v4, idx, bmin, bmax, density=5.0, exact=True) -> Built:
    """Uniform grid (UGridSortBuilder.h:64-407, exact insertion UniformGridBuildKernels.cu:224-383)."""
    v4 = np.ascontiguousarray(v4, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    g = Grid()
    cells = C.c_void_p()
    prims = C.c_void_p()
    np_ = C.c_uint32()
    rc = lib().orc_build_ug(_p(v4), _p(idx), idx.shape[0], _p(np.asarray(bmin, np.float32)),
                            _p(np.asarray(bmax, np.float32)), density, int(exact), C.byref(g),
                            C.byref(cells), C.byref(prims), C.byref(np_))
    if rc != 0:
        raise MemoryError("oracle build_ug failed")
    c = _take(cells, 2 * g.ncells).reshape(-1, 2)
    p = _take(prims, np_.value)
    return Built(UG, v4, idx, g, c, None, p, np_.value)


def build_tl(v4, idx, bmin, bmax, top=0.0625, leaf=2.0) -> Built:
    """Two-level grid (TLGridSortBuilder.h:66-452)."""
    v4 = np.ascontiguousarray(v4, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    g = Grid()
    cells = C.c_void_p()
    leaves = C.c_void_p()
    prims = C.c_void_p()
    nl = C.c_uint32()
    np_ = C.c_uint32()
    ntp = C.c_uint32()
    rc = lib().orc_build_tl(_p(v4), _p(idx), idx.shape[0], _p(np.asarray(bmin, np.float32)),
                            _p(np.asarray(bmax, np.float32)), top, leaf, C.byref(g), C.byref(cells),
                            C.byref(leaves), C.byref(nl), C.byref(prims), C.byref(np_), C.byref(ntp))
    if rc != 0:
        raise MemoryError("oracle build_tl failed")
    c = _take(cells, 2 * g.ncells).reshape(-1, 2)
    lv = _take(leaves, 2 * nl.value).reshape(-1, 2)
    p = _take(prims, np_.value)
    return Built(TL, v4, idx, g, c, lv, p, np_.value, ntp.value)


def camera(pos, fwd, up, fov, w, h) -> Camera:
    cam = Camera()
    lib().orc_camera_init(C.byref(cam), _f3(pos), _f3(fwd), _f3(up), fov, w, h)
    return cam


def primary_rays(cam: Camera):
    n = cam.w * cam.h
    org = np.empty((n, 3), np.float32)
    d = np.empty((n, 3), np.float32)
    lib().orc_primary_rays(C.byref(cam), _p(org), _p(d))
    return org, d


def trace(b: Built, org, dirs, stats=False):
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    n = org.shape[0]
    hid = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    u = np.empty(n, np.float32)
    v = np.empty(n, np.float32)
    st = np.empty((n, 2), np.uint32) if stats else None
    s = b.scene()
    lib().orc_trace(C.byref(s), _p(org), _p(dirs), n, _p(hid), _p(t), _p(u), _p(v), _p(st))
    return (hid, t, u, v, st) if stats else (hid, t, u, v)


def trace_primary(b: Built, cam: Camera, stats=False):
    n = cam.w * cam.h
    hid = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    u = np.empty(n, np.float32)
    v = np.empty(n, np.float32)
    st = np.empty((n, 2), np.uint32) if stats else None
    s = b.scene()
    lib().orc_trace_primary(C.byref(s), C.byref(cam), _p(hid), _p(t), _p(u), _p(v), _p(st))
    return (hid, t, u, v, st) if stats else (hid, t, u, v)


def occluded(b: Built, org, dirs, tmax):
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    tmax = np.ascontiguousarray(tmax, np.float32)
    n = org.shape[0]
    occ = np.empty(n, np.uint8)
    s = b.scene()
    lib().orc_occluded(C.byref(s), _p(org), _p(dirs), _p(tmax), n, _p(occ))
    return occ


def render_ao(b: Built, cam: Camera, spp: int, alpha: float, seed: int, image_id: int = 0,
              fb=None, pixel_stride: int = 1):
    n = cam.w * cam.h
    fb = np.zeros(n, np.float32) if fb is None else np.ascontiguousarray(fb, np.float32)
    counts = np.zeros(1, np.uint64)
    s = b.scene()
    lib().orc_render_ao(C.byref(s), C.byref(cam), spp, alpha, seed, image_id, _p(fb), pixel_stride, _p(counts))
    return fb, int(counts[0])


def render_primary(b: Built, cam: Camera, image_id: int, seed: int, fb=None):
    """Render mode 0 (pixel samplers + simpleShade), blended into fb (pixels x 3 floats)."""
    n = cam.w * cam.h
    fb = np.zeros((n, 3), np.float32) if fb is None else np.ascontiguousarray(fb, np.float32).reshape(n, 3)
    s = b.scene()
    lib().orc_render_primary(C.byref(s), C.byref(cam), image_id, seed, _p(fb))
    return fb


def render_rays(b: Built, org, dirs, image_id: int = 0, fb=None):
    """Ray-file form of render mode 0: ray i traced and shaded into pixel i (n x 3 floats)."""
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    n = org.shape[0]
    fb = np.zeros((n, 3), np.float32) if fb is None else np.ascontiguousarray(fb, np.float32).reshape(n, 3)
    s = b.scene()
    lib().orc_render_rays(C.byref(s), _p(org), _p(dirs), n, image_id, _p(fb))
    return fb


def log_series(x: float) -> float:
    return float(lib().orc_log_series(x))


def render_pt(b: Built, cam: Camera, light, bounces: int, albedo: float, ray_eps: float, seed: int,
              image_id: int = 0, fb=None, pixel_stride: int = 1):
    """Path-traced frame; `light` is one Light or a sequence of them (a light collection)."""
    lights = [light] if isinstance(light, Light) else list(light)
    arr = (Light * len(lights))(*lights)
    n = cam.w * cam.h
    fb = np.zeros(n, np.float32) if fb is None else np.ascontiguousarray(fb, np.float32)
    counts = np.zeros(1, np.uint64)
    s = b.scene()
    lib().orc_render_pt(C.byref(s), C.byref(cam), arr, len(lights), bounces, albedo, ray_eps, seed, image_id,
                        _p(fb), pixel_stride, _p(counts))
    return fb, int(counts[0])


def make_light(corner=(0.4, 0.4, 1.0), e1=(0.2, 0.0, 0.0), e2=(0.0, 0.2, 0.0), emission=20.0,
               normal=(0.0, 0.0, -1.0)) -> Light:
    l = Light()
    l.corner = _f3(corner)
    l.e1 = _f3(e1)
    l.e2 = _f3(e2)
    l.normal = _f3(normal)
    l.emission = emission
    return l


def brute_f64(v4, idx, org, dirs):
    """FP64 brute-force closest hit; flags: 1 t-tie, 2 near edge, 4 grazing."""
    v4 = np.ascontiguousarray(v4, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    n = org.shape[0]
    hid = np.empty(n, np.int32)
    t = np.empty(n, np.float64)
    u = np.empty(n, np.float64)
    v = np.empty(n, np.float64)
    fl = np.empty(n, np.uint8)
    lib().orc_brute_f64(_p(v4), _p(idx), idx.shape[0], _p(org), _p(dirs), n, _p(hid), _p(t), _p(u), _p(v), _p(fl))
    return hid, t, u, v, fl


def sincos2pi(u: float):
    s = C.c_float()
    c = C.c_float()
    lib().orc_sincos2pi(u, C.byref(s), C.byref(c))
    return s.value, c.value


def pcg32_floats(initstate: int, initseq: int, k: int):
    out = np.empty(k, np.float32)
    lib().orc_pcg32_first_floats(initstate, initseq, k, _p(out))
    return out


# ---- instanced two-level grid hierarchy -------------------------------------------

INST_DTYPE = np.dtype([("obj", "<u4"), ("m", "<f4", 12), ("bmin", "<f4", 3), ("bmax", "<f4", 3)])


class BuiltHier:
    """Result of an oracle hierarchy build (TLGridHierarchySortBuilder.cu:373-682); keeps
    the arrays alive for traversal calls."""

    def __init__(self, v4, idx, objs, inst, top, obj_cells, prims, top_cells, inst_ids):
        self.v4, self.idx, self.objs, self.inst, self.top = v4, idx, objs, inst, top
        self.obj_cells, self.prims, self.top_cells, self.inst_ids = obj_cells, prims, top_cells, inst_ids

    def struct(self) -> Hier:
        h = Hier()
        h.v4, h.idx = _p(self.v4), _p(self.idx)
        h.ntri, h.nobj, h.ninst = self.idx.shape[0], len(self.objs), self.inst.shape[0]
        h.objs = C.cast(self.objs, C.c_void_p)
        h.inst = _p(self.inst)
        h.top = self.top
        h.top_cells, h.inst_ids = _p(self.top_cells), _p(self.inst_ids)
        h.obj_cells, h.prims = _p(self.obj_cells), _p(self.prims)
        return h


def hier_build(v, idx, obj_tri_counts, inst, top=1.2, leaf=1.2) -> BuiltHier:
    """Object grids (one uniform grid per object: a consecutive triangle range) and the
    instance grid.  v: (nv, 3) object-space vertices; inst: INST_DTYPE records."""
    v = np.asarray(v, np.float32)
    v4 = np.zeros((v.shape[0], 4), np.float32)
    v4[:, :3] = v
    idx = np.ascontiguousarray(idx, np.uint32)
    counts = np.ascontiguousarray(obj_tri_counts, np.uint32)
    inst = np.ascontiguousarray(inst, INST_DTYPE)
    objs = (Obj * len(counts))()
    g = Grid()
    oc, pr, tc, ii = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    noc, np_, ntp = C.c_uint32(), C.c_uint32(), C.c_uint32()
    rc = lib().orc_hier_build(_p(v4), _p(idx), idx.shape[0], _p(counts), len(counts), _p(inst), inst.shape[0],
                              top, leaf, C.cast(objs, C.c_void_p), C.byref(g), C.byref(oc), C.byref(noc),
                              C.byref(pr), C.byref(np_), C.byref(tc), C.byref(ii), C.byref(ntp))
    if rc != 0:
        raise ValueError("oracle hier_build failed (object triangle counts must sum to the triangle count)")
    return BuiltHier(v4, idx, objs, inst, g, _take(oc, 2 * noc.value).reshape(-1, 2), _take(pr, np_.value),
                     _take(tc, 2 * g.ncells).reshape(-1, 2), _take(ii, ntp.value))


def hier_trace(h: BuiltHier, org, dirs, tmax=None, anyhit=False):
    """Closest hit (instance id, triangle id, t, u, v), or any hit below tmax."""
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    n = org.shape[0]
    tm = None if tmax is None else np.ascontiguousarray(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
    out = [np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32),
           np.empty(n, np.float32)]
    s = h.struct()
    lib().orc_hier_trace(C.byref(s), _p(org), _p(dirs), _p(tm), n, 1 if anyhit else 0, *[_p(a) for a in out])
    return tuple(out)
