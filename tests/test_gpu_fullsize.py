"""Parity at the full sizes of the benchmark configurations.

The other GPU tests use small scenes; the timed workloads are much larger, and the
machinery that only large scenes reach -- capacity fitting, digit-width planning of the
sorts, overflow and regrow, replay of the captured build graph across frame times, the
batch planner over hundreds of scenes -- is checked here on exactly the inputs the
benchmark times:

  c2  1,048,576 triangles, two-level grid 1/16 : 2, 1920x1080 camera rays + 8 AO rays per
      hit: grid and AO image bit-equal to the oracle;
  c3  2,097,152 triangles, 16 curl-noise key frames, several frame times through the
      replayed build graph: every grid bit-equal to the oracle, and the 1280x720 4-bounce
      path-traced image at the last of them;
  c4  256 batched scenes (21.5M triangles): every scene's grid and image bit-identical to
      the per-scene path, the five largest also against the oracle.
"""
import numpy as np
import pytest

from happyray_b200 import GRID_TWO_LEVEL, RENDER_AO, RENDER_PATH, Engine
from happyray_b200 import scenes as S

from tests.test_gpu_parity import assert_same_grid, ocam, oracle_build, set_cam

pytestmark = pytest.mark.gpu

BENCH_SEED = 0x853c49e6748fea9b


@pytest.fixture(scope="module")
def big_engine(hrlib):
    e = Engine(0)
    yield e
    e.cleanup()


def test_c2_full_grid_and_ao_frame(big_engine, oracle):
    e = big_engine
    v, f = S.config_scene("c2")
    assert f.shape[0] == 1_048_576
    e.set_keyframes(v[None], f)
    e.setGridDensities(0.0625, 2.0)
    for _ in range(3):   # the third build replays the captured graph
        e.set_frame_time(0.0, 0.0)
        e.build(GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    assert_same_grid(e.grid_download(), b)
    cam = S.camera_at_bounds(v, (1920, 1080))
    set_cam(e, cam)
    alpha = float(np.float32(0.1) * b.diag())
    e.set_integrator(ao_samples=8, ao_radius=alpha, seed=BENCH_SEED)
    e.ray_count(reset=True)
    fb = e.renderFrame(None, 0, RENDER_AO)
    rays = e.ray_count(reset=True)
    img, orays = oracle.render_ao(b, ocam(oracle, cam), 8, alpha, BENCH_SEED)
    assert rays == orays
    mism = int((fb[:, 0] != img).sum())
    assert mism == 0, f"{mism} of {img.size} AO pixels differ"
    assert np.array_equal(fb[:, 1], img) and np.array_equal(fb[:, 2], img)


def test_c3_full_keyframes_replayed_graph_and_pt_frame(big_engine, oracle):
    e = big_engine
    v, f = S.config_scene("c3")
    assert f.shape[0] == 2_097_152
    frames = S.curl_keyframes_torch(v, 16, amp=0.02, octaves=4, seed=0)
    e.set_keyframes(frames, f)
    e.setGridDensities(0.0625, 2.0)
    # frame times of the 120-step cycle; from the third build on the rebuild replays one
    # captured graph whose interpolation reads the frame pair and weight from device memory
    ks = [0, 1, 37, 74, 95, 119]
    b = None
    for k in ks:
        tt = 16.0 * k / 120.0
        e.set_frame_time(tt, 0.0)
        e.build(GRID_TWO_LEVEL)
        a = int(np.float32(tt))
        c = np.float32(tt) - np.float32(a)
        v4, bmin, bmax = oracle.lerp_bounds(frames[a], frames[(a + 1) % 16], float(c))
        assert np.array_equal(e.vertices(v.shape[0]), v4), f"frame time {tt}"
        b = oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)
        assert_same_grid(e.grid_download(), b)
    cam = S.camera_at_bounds(v, (1280, 720))
    set_cam(e, cam)
    e.set_integrator(pt_bounces=4, albedo=0.7, seed=BENCH_SEED)
    e.setLights((0.4, 0.4, 1.0), (0.2, 0.0, 0.0), (0.0, 0.2, 0.0), 20.0)
    e.ray_count(reset=True)
    fb = e.renderFrame(None, 0, RENDER_PATH)
    rays = e.ray_count(reset=True)
    eps = float(np.float32(1e-4) * b.diag())
    img, orays = oracle.render_pt(b, ocam(oracle, cam), oracle.make_light(), 4, 0.7, eps, BENCH_SEED)
    assert rays == orays
    mism = int((fb[:, 0] != img).sum())
    assert mism == 0, f"{mism} of {img.size} PT pixels differ"
    assert img.max() > 0


def test_c4_full_batch_against_per_scene_and_oracle(hrlib, oracle):
    from happyray_b200.batch import Batch, SceneSpec
    from tests.test_gpu_batch import plain, same_grid
    import tests.test_gpu_batch as TB

    raw = S.batch_scenes(256, 0)
    specs = [SceneSpec(r["v"], r["f"], r["cam"]["position"], r["cam"]["orientation"], r["cam"]["up"],
                       r["cam"]["fov"], r["cam"]["res_x"], r["cam"]["res_y"], ao_samples=4) for r in raw]
    assert sum(s.faces.shape[0] for s in specs) > 20_000_000
    with Batch(0) as bt:
        bt.set_scenes(specs)
        bt.set_integrator(0.1, TB.SEED)
        bt.run(0)
        for i, sp in enumerate(specs):
            pgrid, pimg = plain(sp)
            same_grid(bt.grid_download(i), pgrid)
            assert np.array_equal(bt.image(i), pimg), f"scene {i}"
        largest = sorted(range(len(specs)), key=lambda k: specs[k].faces.shape[0])[-5:]
        for i in largest:
            sp = specs[i]
            ob = oracle_build(oracle, sp.vertices, sp.faces, GRID_TWO_LEVEL)
            gi = bt.grid_info(i)
            for k in ("bounds_min", "bounds_max", "cell_size", "cell_size_rcp"):
                gi[k] = np.array(gi[k], np.float32)
            assert_same_grid((gi,) + tuple(bt.grid_download(i)), ob)
            oc = oracle.camera(sp.position, sp.orientation, sp.up, sp.fov, sp.width, sp.height)
            img, _ = oracle.render_ao(ob, oc, 4, float(np.float32(0.1) * ob.diag()), TB.SEED)
            assert np.array_equal(bt.image(i)[..., 0].reshape(-1), img), f"scene {i} vs oracle"
