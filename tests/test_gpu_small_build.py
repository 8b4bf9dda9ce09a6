"""GPU: the single-launch uniform build of small scenes (build_small.cu) against the build
pipeline and the oracle.  A context created with HAPPYRAY_SMALL_BUILD_MAX_TRIS=0 always
runs the pipeline (lerp, count, scan, scatter, radix passes, ranges as separate kernels);
the default context runs small scenes (at most 131,072 triangles, one 256-thread block
per 256 triangles, at most half the blocks the GPU holds at once) as one cooperative
launch.  Both must give the oracle's
grid bit for bit: cells, primitive lists, bounds, resolution and cell sizes
(UniformGridBuildKernels.h:40-487, Sort.cu:31-53)."""
import functools
import os

import numpy as np
import pytest

from happyray_b200 import GRID_UNIFORM
from happyray_b200 import scenes as S

from test_gpu_parity import assert_same_grid, oracle_build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pipeline_engine(hrlib):
    from happyray_b200 import Engine
    old = os.environ.get("HAPPYRAY_SMALL_BUILD_MAX_TRIS")
    os.environ["HAPPYRAY_SMALL_BUILD_MAX_TRIS"] = "0"
    try:
        e = Engine(0)
    finally:
        if old is None:
            del os.environ["HAPPYRAY_SMALL_BUILD_MAX_TRIS"]
        else:
            os.environ["HAPPYRAY_SMALL_BUILD_MAX_TRIS"] = old
    yield e
    e.cleanup()


def big_triangles(n=100, seed=5):
    """n triangles spanning most of the unit cube: their bounding boxes cover nearly every
    cell, so the first pair estimate (6 per triangle) overflows and the build grows and
    runs again."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(0.0, 1.0, (3 * n, 3)).astype(np.float32)
    v[0::3] = rng.uniform(0.0, 0.1, (n, 3))
    v[1::3] = rng.uniform(0.9, 1.0, (n, 3))
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return v, f


NAMES = ["heightfield_32k", "clusters_60k", "clusters_5k", "two_triangles", "big_triangles"]


@functools.lru_cache(maxsize=None)
def scenes():
    hv, hf = S.heightfield(129, 0)
    cv, cf = S.clusters(60_000, seed=3)
    sv, sf = S.clusters(5_000, seed=7)
    tv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [0.5, 0.2, 0.9]], np.float32)
    tf = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    bv, bf = big_triangles()
    return {"heightfield_32k": (hv, hf), "clusters_60k": (cv, cf), "clusters_5k": (sv, sf),
            "two_triangles": (tv, tf), "big_triangles": (bv, bf)}


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("name", NAMES)
def test_small_build_matches_pipeline_and_oracle(engine, pipeline_engine, oracle, name, exact):
    v, f = scenes()[name]
    want = oracle_build(oracle, v, f, GRID_UNIFORM, exact)
    grids, launches = [], []
    for e in (engine, pipeline_engine):
        e.upload(v, v, f, 1.0)
        e.set_uniform_density(5.0)
        l0 = e.counters()["launches"]
        e.build(GRID_UNIFORM, exact)
        launches.append(e.counters()["launches"] - l0)
        grids.append(e.grid_download())
    for g in grids:
        assert_same_grid(g, want)
    assert launches[1] >= 10
    # Up to 148 * 256 triangles the launch has one block per SM, which qualifies whenever
    # two blocks fit on an SM: the frame selection and one launch per build attempt (the
    # big triangles overflow once and build again).  A larger scene qualifies only while
    # two such launches fit on the GPU at once (60k triangles need 235 blocks) and may
    # take the pipeline instead; its grid is the same either way.
    if f.shape[0] <= 148 * 256:
        assert launches[0] <= 3


def test_small_build_repeated_and_animated(engine, pipeline_engine, oracle):
    """Back-to-back builds reuse the barrier words; resident key frames are interpolated by
    the first phase of the launch and give the pipeline's vertices and grid at every time."""
    v, f = S.clusters(40_000, seed=11)
    frames = S.curl_keyframes(v, 5, seed=2)
    for e in (engine, pipeline_engine):
        e.set_keyframes(frames, f)
        e.set_uniform_density(5.0)
    for tt in [0.0, 1.5, 3.75, 3.75, 0.25, 4.5, 2.0, 2.0, 2.0]:
        grids = []
        for e in (engine, pipeline_engine):
            e.set_frame_time(tt, 0.0)
            e.build(GRID_UNIFORM, True)
            grids.append((e.vertices(v.shape[0]), e.grid_download()))
        k = int(tt)
        c = np.float32(tt) - np.float32(k)
        v4, bmin, bmax = oracle.lerp_bounds(frames[k], frames[(k + 1) % frames.shape[0]], float(c))
        want = oracle.build_ug(v4, f, bmin, bmax, 5.0, True)
        for verts, grid in grids:
            assert np.array_equal(verts, v4)
            assert_same_grid(grid, want)
