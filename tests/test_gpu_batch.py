"""Batched scenes (hr_batch_*): every scene's grid and image from one segmented build and
one persistent render launch must be bit-identical to the per-scene path (hr_ctx) for
the same scene, densities, camera, samples and seed -- and the per-scene path is itself
bit-exact against the oracle (test_gpu_parity.py); one scene is also checked against the
oracle directly here."""
import numpy as np
import pytest

from happyray_b200 import GRID_TWO_LEVEL, RENDER_AO, RENDER_PRIMARY, Engine, HRError
from happyray_b200 import scenes as S
from happyray_b200.batch import Batch, SceneSpec

pytestmark = pytest.mark.gpu

SEED = 0x1234abcd


def make_specs(n=10, seed=5, tri_range=(200, 20_000), px_range=(16 * 16, 72 * 72)):
    raw = S.batch_scenes(n, seed, tri_range, px_range)
    out = []
    for i, r in enumerate(raw):
        cam = r["cam"]
        spp = 0 if i % 3 == 0 else (4 if i % 2 else 8)
        out.append(SceneSpec(r["v"], r["f"], cam["position"], cam["orientation"], cam["up"], cam["fov"],
                             cam["res_x"], cam["res_y"], ao_samples=spp))
    return out


def plain(spec, top=0.0625, leaf=2.0, image_ids=(0,)):
    """The same scene through the per-scene path."""
    e = Engine(0)
    try:
        e.upload(spec.vertices, spec.vertices, spec.faces, 1.0)
        e.setGridDensities(top, leaf)
        e.build(GRID_TWO_LEVEL)
        grid = e.grid_download()
        e.setCamera(spec.position, spec.orientation, spec.up, spec.fov, spec.width, spec.height)
        e.set_integrator(ao_samples=max(spec.ao_samples, 1), ao_radius=-0.1, seed=SEED)
        fb = None
        for im in image_ids:
            fb = e.renderFrame(fb, im, RENDER_AO if spec.ao_samples else RENDER_PRIMARY)
        return grid, fb.reshape(spec.height, spec.width, 3)
    finally:
        e.cleanup()


@pytest.fixture(scope="module")
def specs():
    return make_specs()


@pytest.fixture(scope="module")
def batch(hrlib, specs):
    b = Batch(0)
    b.set_scenes(specs)
    b.set_integrator(0.1, SEED)
    b.run(0)
    yield b
    b.close()


def same_grid(bgrid, pgrid):
    cells, leaves, prims = bgrid
    gi, pc, pl, pp = pgrid
    assert cells.shape == pc.shape and np.array_equal(cells, pc)
    assert leaves.shape == pl.shape and np.array_equal(leaves, pl)
    assert prims.shape == pp.shape and np.array_equal(prims, pp)


def test_batch_grids_match_per_scene(batch, specs):
    for i, sp in enumerate(specs):
        pgrid, _ = plain(sp)
        gi = batch.grid_info(i)
        pgi = pgrid[0]
        assert gi["res"] == pgi["res"]
        assert np.array_equal(np.array(gi["bounds_min"], np.float32), pgi["bounds_min"])
        assert np.array_equal(np.array(gi["cell_size_rcp"], np.float32), pgi["cell_size_rcp"])
        assert (gi["num_cells"], gi["num_leaves"], gi["num_pairs"], gi["num_top_pairs"]) == \
            (pgi["num_cells"], pgi["num_leaves"], pgi["num_pairs"], pgi["num_top_pairs"])
        same_grid(batch.grid_download(i), pgrid)


def test_batch_images_match_per_scene(batch, specs):
    for i, sp in enumerate(specs):
        _, pimg = plain(sp)
        assert np.array_equal(batch.image(i), pimg), f"scene {i}"


def test_batch_grid_matches_oracle(batch, specs, oracle):
    """One scene directly against the CPU oracle (sorted per-cell lists, bit-exact)."""
    i = max(range(len(specs)), key=lambda k: specs[k].faces.shape[0])
    sp = specs[i]
    from tests.test_gpu_parity import assert_same_grid, oracle_build
    b = oracle_build(oracle, sp.vertices, sp.faces, GRID_TWO_LEVEL)
    gi = batch.grid_info(i)
    for k in ("bounds_min", "bounds_max", "cell_size", "cell_size_rcp"):
        gi[k] = np.array(gi[k], np.float32)
    assert_same_grid((gi,) + tuple(batch.grid_download(i)), b)


def test_batch_progressive_and_graph_modes(hrlib, specs):
    sub = specs[:5]
    with Batch(0) as g, Batch(0) as e:
        g.set_scenes(sub)
        e.set_scenes(sub)
        e.set_graph(False)
        for b in (g, e):
            b.set_integrator(0.1, SEED)
            b.run(0)
            b.run(1)
        for i, sp in enumerate(sub):
            _, pimg = plain(sp, image_ids=(0, 1))
            assert np.array_equal(g.image(i), pimg)
            assert np.array_equal(e.image(i), pimg)
        # replaying the same step gives the same image (image 0 overwrites)
        g.run(0)
        _, p0 = plain(sub[1])
        assert np.array_equal(g.image(1), p0)
        c = g.counters()
        assert c[0] > 0 and c[2] == len(sub)
        for b in (g, e):   # build, render and step device times are measured in both modes
            tb, tr, tt = b.times()
            assert tb > 0 and tr > 0 and tt >= tb + tr * 0.99


@pytest.mark.parametrize("shape", [(64, 4), (256, 16), (32, 32)])
def test_batch_launch_shapes_and_densities(hrlib, specs, shape):
    sub = specs[:4]
    with Batch(0) as b:
        b.set_scenes(sub)
        b.set_integrator(0.1, SEED)
        b.set_launch(*shape)
        b.set_densities(0.125, 4.0)
        b.set_densities(0.03125, 1.0, scene=2)
        b.run(0)
        for i, sp in enumerate(sub):
            top, leaf = (0.03125, 1.0) if i == 2 else (0.125, 4.0)
            pgrid, pimg = plain(sp, top, leaf)
            same_grid(b.grid_download(i), pgrid)
            assert np.array_equal(b.image(i), pimg)


def test_batch_autotune(hrlib, specs):
    with Batch(0) as b:
        b.set_scenes(specs[:3])
        best = b.autotune(reps=1)
        assert best["trials"] == 16 + 9
        assert best["ms_per_step"] > 0
        assert best["block_threads"] in (64, 128, 256) and best["tile_width"] in (4, 8, 16)
        b.run(0)


def test_batch_rejects_bad_input(hrlib):
    v, f = S.heightfield(9, 0)
    cam = S.camera_at_bounds(v, (16, 16))
    bad = f.copy()
    bad[3, 1] = v.shape[0]   # out of range of its own scene
    good = SceneSpec(v, f, cam["position"], cam["orientation"], cam["up"], 60.0, 16, 16)
    with Batch(0) as b:
        b.set_integrator(0.1, SEED)
        b.set_scenes([good, SceneSpec(v, bad, cam["position"], cam["orientation"], cam["up"], 60.0, 16, 16)])
        with pytest.raises(HRError) as ei:
            b.run(0)
        assert ei.value.status == 1
        with pytest.raises(HRError):
            b.set_launch(48, 8)
        with pytest.raises(HRError):
            b.set_scenes([SceneSpec(v, f[:0], cam["position"], cam["orientation"], cam["up"], 60.0, 16, 16)])
        # a valid set after the failures works
        b.set_scenes([good])
        b.run(0)
        _, pimg = plain(good)
        assert np.array_equal(b.image(0), pimg)
