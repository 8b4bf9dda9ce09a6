"""The RTEngine adapter (happyray_b200/adapter/RTEngine.cu): the reference's engine facade
implemented on the C-ABI, as a maintainer drops it into the reference project.

CPU: it implements every method RTEngine.h declares, and it compiles against the
reference's own headers (when the reference's source tree is present).
GPU (test_gpu_adapter_* below): the harness drives it with the reference's WFObject,
AreaLightSourceCollection and FrameBuffer classes, and every frame equals the library's
own calls on the same inputs, bit for bit."""
import os
import re
import struct
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
ADAPTER = ROOT / "happyray_b200" / "adapter"
HARNESS = ADAPTER / "_bin" / "rtengine_harness"
sys.path.insert(0, str(ROOT))


def reference_tree():
    from __graft_entry__ import reference_tree as rt
    return rt()


# the methods of src/RT/RTEngine.h:36-68
RTENGINE_METHODS = ["init", "upload", "buildAccStruct", "setCamera", "setLights", "renderFrame", "setGridDensities",
                    "cleanup", "getBoundingBoxDiagonalLength", "setInputRayFileName"]


def test_adapter_defines_every_rtengine_method():
    src = ADAPTER.joinpath("RTEngine.cu").read_text()
    for m in RTENGINE_METHODS:
        assert re.search(r"\bRTEngine::%s\s*\(" % m, src), m
    header = reference_tree() / "src" / "RT" / "RTEngine.h"
    if header.exists():   # the header itself lists exactly these
        declared = re.findall(r"static\s+[\w:&<>\s]+?\b(\w+)\s*\(", header.read_text())
        assert sorted(declared) == sorted(RTENGINE_METHODS)


def test_adapter_compiles_against_reference_headers(tmp_path):
    tree = reference_tree()
    if not (tree / "src" / "RT" / "RTEngine.h").exists():
        pytest.skip("the reference's source tree is not present")
    r = subprocess.run(["make", "-s", "-C", str(ADAPTER), f"REF={tree.resolve()}", f"OUT={tmp_path}",
                        f"{tmp_path}/RTEngine.o"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert (tmp_path / "RTEngine.o").stat().st_size > 0


# -- GPU: a frame through the adapter equals the library's own calls --------------------------

def harness_input(path, v1, v2, faces, coeff, dens, cam, lights, ray_file=""):
    with open(path, "wb") as f:
        f.write(b"HRA1")
        f.write(struct.pack("<II", v1.shape[0], faces.shape[0]))
        f.write(struct.pack("<fff", coeff, dens[0], dens[1]))
        f.write(np.asarray(list(cam["position"]) + list(cam["orientation"]) + list(cam["up"]), np.float32).tobytes())
        f.write(struct.pack("<fii", cam["fov"], cam["res_x"], cam["res_y"]))
        f.write(struct.pack("<I", len(lights)))
        p = ray_file.encode()
        f.write(struct.pack("<I", len(p)) + p)
        f.write(np.ascontiguousarray(v1, np.float32).tobytes())
        f.write(np.ascontiguousarray(v2, np.float32).tobytes())
        f.write(np.ascontiguousarray(faces, np.uint32).tobytes())
        for L in lights:
            f.write(np.asarray(L, np.float32).reshape(15).tobytes())


@pytest.mark.gpu
def test_gpu_adapter_frames_equal_library_calls(hrlib, tmp_path):
    if not HARNESS.exists():
        pytest.skip("the adapter harness was not built (it needs the reference's source tree at build time)")
    import torch
    from happyray_b200 import GRID_TWO_LEVEL, Engine
    from happyray_b200 import scenes as S
    from happyray_b200 import sceneio
    v, f = S.clusters(20_000, seed=9)
    v2 = (v + np.random.default_rng(9).normal(0, 0.003, v.shape)).astype(np.float32)
    coeff, dens = 0.4, (0.0625, 2.0)
    cam = S.camera_at_bounds(v, (80, 60))
    cam["up"] = (0.0, 0.0, 1.0)
    lights = [[0.4, 0.4, 1.0, 0.2, 0, 0, 0, 0.2, 0, 0, 0, -1, 20, 20, 20],
              [0.1, -0.3, 0.2, 0.6, 0, 0, 0, 0, 0.5, 0, 1, 0, 5, 6, 7]]
    rng = np.random.default_rng(4)
    org = rng.uniform(v.min(0), v.max(0), (3000, 3)).astype(np.float32)
    dirs = rng.normal(size=(3000, 3)).astype(np.float32)
    sceneio.write_rays(str(tmp_path / "q.rays"), org, dirs)
    harness_input(tmp_path / "in.bin", v, v2, f, coeff, dens, cam, lights, str(tmp_path / "q.rays"))
    r = subprocess.run([str(HARNESS), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(tmp_path / "out.bin", np.float32)
    npx = cam["res_x"] * cam["res_y"]
    diag, rest = out[0], out[1:].reshape(-1, npx, 3)
    assert rest.shape[0] == 4
    # the same frames through the library's own calls (the settings the adapter's init makes)
    with Engine(0) as e:
        e.upload(v, v2, f, coeff)
        e.setGridDensities(*dens)
        e.build(GRID_TWO_LEVEL)
        e.setCamera(cam["position"], cam["orientation"], cam["up"], cam["fov"], cam["res_x"], cam["res_y"])
        L = np.asarray(lights, np.float32)
        e.setLights(L[:, 0:3], L[:, 3:6], L[:, 6:9], L[:, 12:15].mean(axis=1), normals=L[:, 9:12])
        e.set_integrator(ao_samples=4, ao_radius=-0.05, pt_bounces=4, albedo=0.7, seed=0x853c49e6748fea9b)
        assert np.float32(e.getBoundingBoxDiagonalLength()) == diag
        fb = None
        for im in range(6):
            fb = e.renderFrame(fb, im, 0)
        assert np.array_equal(rest[0], fb.reshape(npx, 3))
        assert np.array_equal(rest[1], e.renderFrame(None, 0, 3).reshape(npx, 3))
        assert np.array_equal(rest[2], e.renderFrame(None, 0, 1).reshape(npx, 3))
        d_org = torch.from_numpy(org).cuda()
        d_dir = torch.from_numpy(dirs).cuda()
        d_fb = torch.zeros((org.shape[0], 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        e.render_rays_device(d_org, d_dir, org.shape[0], 0, d_fb)
        e.sync()
        assert np.array_equal(rest[3][:org.shape[0]], d_fb.cpu().numpy())
        assert np.all(rest[3][org.shape[0]:] == 0)
