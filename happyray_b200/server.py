"""Served rendering over the C-ABI (hr_server_* in include/happyray.h).

A Server keeps animated scenes resident and answers render and ray-query requests.  In
batched mode its worker thread admits queued requests under the HBM budget, rebuilds a
scene's grid only when a request asks for another frame time, and traces every admitted
request of a wave in one persistent launch, with two waves in flight.  Serial mode runs
the same requests one at a time through the per-scene path on the resident scenes; plain
mode is the drop-in per-frame path (one context; per request upload the frame, build,
render, read back).  Results do not depend on the mode or on the other requests.  The
reference has no server: its application renders one scene per process
(src/Application/CUDAApplication.cu:116-160).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import HRError, Request, RequestInfo, ServerStats

BATCHED, SERIAL, PLAIN = 0, 1, 2
RENDER, RAYS = 0, 1


class Pending:
    """A submitted request and the buffers it writes (kept alive until it is done)."""

    def __init__(self, server: "Server", rid: int, out, keep):
        self.server = server
        self.id = rid
        self.out = out
        self._keep = keep

    def wait(self, timeout_ms: int = -1):
        self.server._chk(self.server.L.hr_server_wait(self.server.s, self.id, timeout_ms), "wait")
        return self.out

    def info(self) -> dict:
        i = RequestInfo()
        self.server._chk(self.server.L.hr_server_request_info(self.server.s, self.id, C.byref(i)), "request_info")
        return {"status": i.status, "wave": i.wave, "submit_ns": i.submit_ns, "admit_ns": i.admit_ns,
                "done_ns": i.done_ns}


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 120 << 30, mode: int = BATCHED):
        self.L = _lib.load()
        s = C.c_void_p()
        st = self.L.hr_server_create(C.byref(s), device, int(hbm_budget_bytes), mode)
        if st != 0:
            raise HRError(st, f"hr_server_create(device={device}) failed")
        self.s = s
        self.mode = mode

    def close(self):
        if getattr(self, "s", None):
            self.L.hr_server_destroy(self.s)
            self.s = None

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
            m = self.L.hr_server_last_error(self.s)
            raise HRError(st, f"{what}: {m.decode() if m else ''}")

    def add_scene(self, keyframes: np.ndarray, faces: np.ndarray, top_density: float = 0.0625,
                  leaf_density: float = 2.0) -> int:
        kf = np.ascontiguousarray(keyframes, np.float32)
        if kf.ndim == 2:
            kf = kf[None]
        f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
        sid = C.c_uint32()
        self._chk(self.L.hr_server_add_scene(self.s, kf.ctypes.data, kf.shape[0], kf.shape[1], f.ctypes.data,
                                             f.shape[0], top_density, leaf_density, C.byref(sid)), "add_scene")
        return sid.value

    def submit_render(self, scene: int, frame_time: float, mode: int, spp: int, cam: dict, seed: int,
                      out: Optional[np.ndarray] = None) -> Pending:
        """cam: position, orientation, up, fov, res_x, res_y (scenes.camera_* dicts)."""
        w, h = int(cam["res_x"]), int(cam["res_y"])
        if out is None:
            out = np.zeros((h * w, 3), np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != w * h * 3:
            raise HRError(1, "submit_render: out must be contiguous float32 with 3 floats per pixel")
        r = Request()
        r.scene, r.frame_time, r.kind, r.mode, r.spp = scene, frame_time, RENDER, mode, spp
        r.cam_position[:] = [float(x) for x in cam["position"]]
        r.cam_orientation[:] = [float(x) for x in cam["orientation"]]
        r.cam_up[:] = [float(x) for x in cam["up"]]
        r.cam_fov_deg = float(cam["fov"])
        r.width, r.height = w, h
        r.seed = seed
        r.out_rgb = out.ctypes.data
        rid = C.c_uint64()
        self._chk(self.L.hr_server_submit(self.s, C.byref(r), C.byref(rid)), "submit")
        return Pending(self, rid.value, out, [out])

    def submit_rays(self, scene: int, frame_time: float, org: np.ndarray, dirs: np.ndarray, outs=None) -> Pending:
        o = np.ascontiguousarray(org, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        n = o.shape[0]
        if outs is None:
            outs = (np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32))
        r = Request()
        r.scene, r.frame_time, r.kind = scene, frame_time, RAYS
        r.ray_org, r.ray_dir, r.num_rays = o.ctypes.data, d.ctypes.data, n
        r.out_id, r.out_t, r.out_u, r.out_v = [a.ctypes.data for a in outs]
        rid = C.c_uint64()
        self._chk(self.L.hr_server_submit(self.s, C.byref(r), C.byref(rid)), "submit")
        return Pending(self, rid.value, outs, [o, d, outs])

    def drain(self, timeout_ms: int = -1):
        self._chk(self.L.hr_server_drain(self.s, timeout_ms), "drain")

    def set_watchdog(self, timeout_ms: int):
        """Requests of a wave still unfinished timeout_ms after its launch fail with
        HR_ERR_TIMEOUT (0: off)."""
        self._chk(self.L.hr_server_set_watchdog(self.s, int(timeout_ms)), "set_watchdog")

    def inject_stall(self, waves: int, stall_ms: int):
        """Test hook: the next `waves` waves are held back stall_ms on the host."""
        self._chk(self.L.hr_server_inject_stall(self.s, int(waves), int(stall_ms)), "inject_stall")

    def stats(self) -> dict:
        st = ServerStats()
        self._chk(self.L.hr_server_get_stats(self.s, C.byref(st)), "stats")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}
