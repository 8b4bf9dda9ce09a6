"""The fast-arithmetic build (libhappyray_b200_fast.so): the traversal kernels compiled with
FMA contraction, approximate division and square root, the grid build left IEEE.  Its
results are held to the floating-point tolerance of the ray queries instead of bit
equality: ray ids equal to the FP64 brute force except at flagged ties, t, u and v within
1e-5 relative (RayTriangleIntersector.h:52-90 evaluated in binary64), grids bit-exact, and
rendered images within the stated bounds of the oracle's."""
import numpy as np
import pytest

from happyray_b200 import GRID_TWO_LEVEL, GRID_UNIFORM, RENDER_AO, RENDER_PATH
from happyray_b200 import scenes as S

from tests.test_gpu_parity import assert_same_grid, gpu_build, ocam, oracle_build, set_cam
from tests.test_oracle import compare_fp64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fast_engine():
    from happyray_b200 import Engine, _lib
    from happyray_b200 import build as B
    if not B.OUT_FAST.exists():
        B.build(fast=True)
    e = Engine(0, lib=_lib.load_fast())
    yield e
    e.cleanup()


@pytest.mark.parametrize("kind", [GRID_UNIFORM, GRID_TWO_LEVEL])
def test_fast_ray_queries_within_fp64_tolerance(fast_engine, oracle, small_clusters, kind):
    v, f = small_clusters
    assert_same_grid(gpu_build(fast_engine, v, f, kind), oracle_build(oracle, v, f, kind))
    cam = S.camera_at_bounds(v, (320, 240))
    org, d = oracle.primary_rays(ocam(oracle, cam))
    rng = np.random.default_rng(7)
    org2 = rng.uniform(v.min(0), v.max(0), (3000, 3)).astype(np.float32)
    d2 = rng.normal(size=(3000, 3)).astype(np.float32)
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    org = np.concatenate([org, org2])
    d = np.concatenate([d, d2])
    hid, t, u, vv = fast_engine.trace_rays(org, d)
    v4, _, _ = oracle.lerp_bounds(v, v, 1.0)
    sel = np.random.default_rng(1).choice(org.shape[0], 3000, replace=False)
    frac, nhit = compare_fp64(oracle, v4, f, org[sel], d[sel], hid[sel], t[sel], u[sel], vv[sel])
    assert frac > 0.99 and nhit > 500


def test_fast_ao_and_pt_images_near_oracle(fast_engine, oracle, small_clusters):
    """AO: a pixel's visibility is a count of free rays out of 8, so a sample ray whose
    hit decision flips at a grazing or near-tangent intersection changes it by 1/8; at most
    1% of the pixels may differ and the mean absolute difference stays under 2e-3.  PT:
    a flipped decision sends the rest of that path elsewhere, so only the image mean is
    held (within 1%)."""
    v, f = small_clusters
    gpu_build(fast_engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    cam = S.camera_at_bounds(v, (160, 120))
    set_cam(fast_engine, cam)
    alpha = float(np.float32(0.1) * b.diag())
    fast_engine.set_integrator(ao_samples=8, ao_radius=alpha, seed=5)
    fb = fast_engine.renderFrame(None, 0, RENDER_AO)
    img, _ = oracle.render_ao(b, ocam(oracle, cam), 8, alpha, 5)
    dif = np.abs(fb[:, 0].astype(np.float64) - img)
    assert (dif > 0).mean() <= 0.01 and dif.mean() <= 2e-3, ((dif > 0).mean(), dif.mean())
    fast_engine.set_integrator(pt_bounces=4, albedo=0.7, seed=11)
    fast_engine.setLights((0.4, 0.4, 1.0), (0.2, 0, 0), (0, 0.2, 0), 20.0)
    fb = fast_engine.renderFrame(None, 0, RENDER_PATH)
    eps = float(np.float32(1e-4) * b.diag())
    img, _ = oracle.render_pt(b, ocam(oracle, cam), oracle.make_light(), 4, 0.7, eps, 11)
    assert abs(fb[:, 0].mean() - img.mean()) <= 0.01 * img.mean(), (fb[:, 0].mean(), img.mean())
