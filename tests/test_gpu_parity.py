"""GPU parity: the CUDA library (through the C-ABI) against the CPU oracle on the same
inputs.  Integer results (cells, leaves, primitive lists, hit ids) and the float results
(t, u, v, AO / PT pixels) are compared bit-exact: both sides evaluate the same binary32
expressions in the same order without FMA contraction.  t/u/v are additionally held to
1e-5 relative against the FP64 brute-force oracle (see test_oracle.compare_fp64)."""
from pathlib import Path

import numpy as np
import pytest

from happyray_b200 import GRID_TWO_LEVEL, GRID_UNIFORM, RENDER_AO, RENDER_PATH, RENDER_PRIMARY
from happyray_b200 import scenes as S

pytestmark = pytest.mark.gpu


def oracle_build(O, v, f, kind, exact=True, ug=5.0, top=0.0625, leaf=2.0):
    v4, bmin, bmax = O.lerp_bounds(v, v, 1.0)
    if kind == GRID_UNIFORM:
        return O.build_ug(v4, f, bmin, bmax, ug, exact)
    return O.build_tl(v4, f, bmin, bmax, top, leaf)


def gpu_build(e, v, f, kind, exact=True, ug=5.0, top=0.0625, leaf=2.0, coeff=1.0, v2=None):
    e.upload(v, v if v2 is None else v2, f, coeff)
    e.set_uniform_density(ug)
    e.setGridDensities(top, leaf)
    e.build(kind, exact)
    return e.grid_download()


def assert_same_grid(gpu, orc):
    gi, cells, leaves, prims = gpu
    g = orc.grid
    assert gi["res"] == tuple(g.res)
    assert np.array_equal(gi["bounds_min"], np.array(g.bmin, np.float32))
    assert np.array_equal(gi["bounds_max"], np.array(g.bmax, np.float32))
    assert np.array_equal(gi["cell_size"], np.array(g.cs, np.float32))
    assert np.array_equal(gi["cell_size_rcp"], np.array(g.rcp, np.float32))
    assert gi["num_cells"] == g.ncells
    assert gi["num_pairs"] == orc.npairs
    assert np.array_equal(cells, orc.cells)
    if orc.leaves is not None:
        assert gi["num_top_pairs"] == orc.ntop_pairs
        assert np.array_equal(leaves, orc.leaves)
    assert np.array_equal(prims, orc.prims)


def ocam(O, cam):
    return O.camera(cam["position"], cam["orientation"], cam["up"], cam["fov"], cam["res_x"], cam["res_y"])


def set_cam(e, cam):
    e.setCamera(cam["position"], cam["orientation"], cam["up"], cam["fov"], cam["res_x"], cam["res_y"])


@pytest.mark.parametrize("exact", [True, False])
def test_build_uniform_c1(engine, oracle, c1_scene, exact):
    v, f = c1_scene
    assert_same_grid(gpu_build(engine, v, f, GRID_UNIFORM, exact), oracle_build(oracle, v, f, GRID_UNIFORM, exact))


def test_build_two_level_c1(engine, oracle, c1_scene):
    v, f = c1_scene
    assert_same_grid(gpu_build(engine, v, f, GRID_TWO_LEVEL), oracle_build(oracle, v, f, GRID_TWO_LEVEL))


@pytest.mark.parametrize("dens", [(0.0625, 2.0), (1.2, 2.2), (1 / 32, 8.0), (0.25, 1.0)])
def test_build_two_level_clusters(engine, oracle, small_clusters, dens):
    v, f = small_clusters
    assert_same_grid(gpu_build(engine, v, f, GRID_TWO_LEVEL, top=dens[0], leaf=dens[1]),
                     oracle_build(oracle, v, f, GRID_TWO_LEVEL, top=dens[0], leaf=dens[1]))


def test_build_uniform_clusters(engine, oracle, small_clusters):
    v, f = small_clusters
    assert_same_grid(gpu_build(engine, v, f, GRID_UNIFORM, True), oracle_build(oracle, v, f, GRID_UNIFORM, True))


def test_keyframe_lerp_and_rebuild(engine, oracle, small_clusters):
    """Resident key frames, frame-time selection (AnimationManager.hpp:68-97) and the fused
    device interpolation give the oracle's vertices and grid at every frame time.  From the
    third frame on, the rebuilds replay one captured build graph whose lerp kernel reads each
    frame's pair and weight from device memory."""
    v, f = small_clusters
    frames = S.curl_keyframes(v, 6, seed=4)
    engine.set_keyframes(frames, f)
    engine.setGridDensities(0.0625, 2.0)
    for tt, step in [(0.0, 0.0), (2.75, 0.0), (5.5, 0.0), (0.5, 0.0), (3.25, 0.0), (4.75, 0.0), (1.25, 1.0)]:
        engine.set_frame_time(tt, step)
        engine.build(GRID_TWO_LEVEL)
        k = int(tt)
        nxt = (k + 1 + int(step)) % frames.shape[0]
        c = np.float32(tt) - np.float32(k)
        v4, bmin, bmax = oracle.lerp_bounds(frames[k], frames[nxt], float(c))
        assert np.array_equal(engine.vertices(v.shape[0]), v4)
        b = oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)
        assert_same_grid(engine.grid_download(), b)


def test_replayed_rebuild_reads_new_vertices_and_recaptures_on_new_settings(engine, oracle, small_clusters):
    """Identical consecutive builds capture the rebuild as a CUDA graph and replay it.  New
    vertices of the same size go into the same buffers, so the next build is a replay: it
    must read them.  Changing the densities, the grid kind or the insertion mode must not
    replay the old graph."""
    v, f = small_clusters
    engine.setGridDensities(0.0625, 2.0)
    engine.upload(v, v, f, 1.0)
    for _ in range(3):
        engine.build(GRID_TWO_LEVEL)
    assert_same_grid(engine.grid_download(), oracle_build(oracle, v, f, GRID_TWO_LEVEL))
    rng = np.random.default_rng(11)
    for k in range(2):
        v2 = (v + rng.normal(0, 0.002, v.shape)).astype(np.float32)
        engine.upload(v2, v2, f, 1.0)
        engine.build(GRID_TWO_LEVEL)
        assert_same_grid(engine.grid_download(), oracle_build(oracle, v2, f, GRID_TWO_LEVEL))
    for top, leaf in [(0.125, 3.0), (0.125, 3.0), (0.125, 3.0), (0.0625, 2.0)]:
        engine.setGridDensities(top, leaf)
        engine.build(GRID_TWO_LEVEL)
        assert_same_grid(engine.grid_download(), oracle_build(oracle, v2, f, GRID_TWO_LEVEL, top=top, leaf=leaf))
    engine.set_uniform_density(5.0)
    for exact in (True, True, True, False, False, False, True):
        engine.build(GRID_UNIFORM, exact)
        assert_same_grid(engine.grid_download(), oracle_build(oracle, v2, f, GRID_UNIFORM, exact))


def test_upload_coefficient(engine, oracle, small_clusters):
    v, f = small_clusters
    v2 = (v + np.random.default_rng(3).normal(0, 0.005, v.shape)).astype(np.float32)
    gpu = gpu_build(engine, v, f, GRID_UNIFORM, True, coeff=0.3, v2=v2)
    v4, bmin, bmax = oracle.lerp_bounds(v, v2, 0.3)
    assert np.array_equal(engine.vertices(v.shape[0]), v4)
    assert_same_grid(gpu, oracle.build_ug(v4, f, bmin, bmax, 5.0, True))


@pytest.mark.parametrize("kind", [GRID_UNIFORM, GRID_TWO_LEVEL])
def test_trace_primary_bitexact_c1(engine, oracle, c1_scene, kind):
    import torch
    v, f = c1_scene
    gpu_build(engine, v, f, kind)
    b = oracle_build(oracle, v, f, kind)
    cam = S.camera_c1()
    set_cam(engine, cam)
    n = 256 * 256
    out = [torch.empty(n, dtype=dt, device="cuda") for dt in (torch.int32, torch.float32, torch.float32, torch.float32)]
    st = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    engine.trace_primary_device(*out, st)
    engine.sync()
    hid, t, u, vv, ost = oracle.trace_primary(b, ocam(oracle, cam), stats=True)
    assert np.array_equal(out[0].cpu().numpy(), hid)
    assert np.array_equal(out[1].cpu().numpy(), t)
    assert np.array_equal(out[2].cpu().numpy(), u)
    assert np.array_equal(out[3].cpu().numpy(), vv)
    assert np.array_equal(st.cpu().numpy().view(np.uint32).reshape(-1, 2), ost)
    assert (hid >= 0).sum() > 10000


@pytest.mark.parametrize("kind", [GRID_UNIFORM, GRID_TWO_LEVEL])
def test_trace_rays_host_api(engine, oracle, small_clusters, kind):
    v, f = small_clusters
    gpu_build(engine, v, f, kind)
    b = oracle_build(oracle, v, f, kind)
    rng = np.random.default_rng(11)
    n = 40000
    org = rng.uniform(-0.2, 1.2, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:50, 1:] = 0.0     # axis-parallel rays (infinite reciprocals)
    d[:50, 0] = 1.0
    got = engine.trace_rays(org, d)
    want = oracle.trace(b, org, d)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)
    from test_oracle import compare_fp64
    sel = slice(0, 3000)
    frac, nhit = compare_fp64(oracle, b.v4, f, org[sel], d[sel], got[0][sel], got[1][sel], got[2][sel], got[3][sel])
    assert frac > 0.98


def test_occluded_matches_oracle(engine, oracle, small_clusters):
    import torch
    v, f = small_clusters
    gpu_build(engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    rng = np.random.default_rng(12)
    n = 30000
    org = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = rng.uniform(0.01, 0.5, n).astype(np.float32)
    want = oracle.occluded(b, org, d, tmax)
    to = lambda a: torch.from_numpy(a).cuda()
    occ = torch.empty(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    engine.occluded_device(to(org), to(d), to(tmax), n, occ)
    engine.sync()
    assert np.array_equal(occ.cpu().numpy(), want)
    assert 0 < want.sum() < n


@pytest.mark.parametrize("kind", [GRID_TWO_LEVEL, GRID_UNIFORM])
def test_render_ao_bitexact(engine, oracle, small_clusters, kind):
    """AO images bit-exact against the oracle: on a two-level grid through the kernel that
    refills lanes inside the traversal loop, on a uniform grid through the one-ray-per-lane
    kernel."""
    v, f = small_clusters
    gpu_build(engine, v, f, kind)
    b = oracle_build(oracle, v, f, kind)
    cam = S.camera_at_bounds(v, (160, 120))
    set_cam(engine, cam)
    alpha = float(np.float32(0.1) * b.diag())
    seed = 1234567
    engine.set_integrator(ao_samples=8, ao_radius=alpha, seed=seed)
    engine.ray_count(reset=True)
    fb = engine.renderFrame(None, 0, RENDER_AO)
    rays = engine.ray_count(reset=True)
    img, orays = oracle.render_ao(b, ocam(oracle, cam), 8, alpha, seed)
    assert np.array_equal(fb[:, 0], img) and np.array_equal(fb[:, 1], img) and np.array_equal(fb[:, 2], img)
    assert rays == orays
    # progressive blend of a second image (AOIntegrator.h:168-175)
    fb2 = engine.renderFrame(fb.copy(), 1, RENDER_AO)
    img2, _ = oracle.render_ao(b, ocam(oracle, cam), 8, alpha, seed, image_id=1, fb=img.copy())
    assert np.array_equal(fb2[:, 0], img2)


def test_render_pt_bitexact(engine, oracle, small_clusters):
    v, f = small_clusters
    gpu_build(engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    cam = S.camera_at_bounds(v, (128, 96))
    set_cam(engine, cam)
    seed = 99
    engine.set_integrator(pt_bounces=4, albedo=0.7, seed=seed)
    engine.setLights((0.4, 0.4, 1.0), (0.2, 0, 0), (0, 0.2, 0), 20.0)
    engine.ray_count(reset=True)
    fb = engine.renderFrame(None, 0, RENDER_PATH)
    rays = engine.ray_count(reset=True)
    eps = float(np.float32(1e-4) * b.diag())
    img, orays = oracle.render_pt(b, ocam(oracle, cam), oracle.make_light(), 4, 0.7, eps, seed)
    assert np.array_equal(fb[:, 0], img)
    assert rays == orays
    assert img.max() > 0


def test_render_pt_light_collection_bitexact(engine, oracle, small_clusters):
    """Two lights through hr_set_lights: a ceiling quad and a wall quad facing +y, picked per
    next-event sample by their weights (area x emission) from the running sum, each
    contribution divided by its probability; the camera sees the emitters directly too."""
    v, f = small_clusters
    gpu_build(engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    cam = S.camera_at_bounds(v, (128, 96))
    set_cam(engine, cam)
    corners = np.array([[0.4, 0.4, 1.0], [0.1, -0.3, 0.2]], np.float32)
    e1 = np.array([[0.2, 0.0, 0.0], [0.6, 0.0, 0.0]], np.float32)
    e2 = np.array([[0.0, 0.2, 0.0], [0.0, 0.0, 0.5]], np.float32)
    normals = np.array([[0.0, 0.0, -1.0], [0.0, 1.0, 0.0]], np.float32)
    em = np.array([20.0, 6.0], np.float32)
    engine.setLights(corners, e1, e2, em, normals=normals)
    seed = 4242
    engine.set_integrator(pt_bounces=4, albedo=0.7, seed=seed)
    engine.ray_count(reset=True)
    fb = engine.renderFrame(None, 0, RENDER_PATH)
    rays = engine.ray_count(reset=True)
    eps = float(np.float32(1e-4) * b.diag())
    lights = [oracle.make_light(corners[k], e1[k], e2[k], float(em[k]), normals[k]) for k in range(2)]
    img, orays = oracle.render_pt(b, ocam(oracle, cam), lights, 4, 0.7, eps, seed)
    assert np.array_equal(fb[:, 0], img)
    assert rays == orays
    # the same collection with a single light equals hr_set_light
    engine.setLights(corners[:1], e1[:1], e2[:1], em[:1], normals=normals[:1])
    one = engine.renderFrame(None, 0, RENDER_PATH)
    engine.setLights(corners[0], e1[0], e2[0], float(em[0]))
    assert np.array_equal(engine.renderFrame(None, 0, RENDER_PATH), one)
    from happyray_b200 import HRError
    for n in (0, 65):
        c = np.tile(corners[:1], (max(n, 1), 1))
        a, bb = np.tile(e1[:1], (max(n, 1), 1)), np.tile(e2[:1], (max(n, 1), 1))
        st = engine.L.hr_set_lights(engine.ctx, n, c.ctypes.data, a.ctypes.data, bb.ctypes.data, None,
                                    np.ones(max(n, 1), np.float32).ctypes.data)
        assert st == 1   # HR_ERR_INVALID_ARG
    with pytest.raises(HRError):   # degenerate: zero-area quad
        engine.setLights(corners, e1, np.zeros_like(e2), em)
    engine.setLights((0.4, 0.4, 1.0), (0.2, 0, 0), (0, 0.2, 0), 20.0)


def test_render_pt_shading_normals_and_materials_bitexact(engine, oracle, small_clusters):
    """Path tracing with per-vertex shading normals (area-weighted vertex normals of the
    mesh, blended at a hit as PathTracer.h:111-136) and a per-triangle albedo table,
    bit-exact against the oracle; removing them gives back the plain images."""
    v, f = small_clusters
    gpu_build(engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    cam = S.camera_at_bounds(v, (96, 72))
    set_cam(engine, cam)
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]]).astype(np.float64)
    vn = np.zeros(v.shape, np.float64)
    for k in range(3):
        np.add.at(vn, f[:, k], fn)
    vn = (vn / np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)).astype(np.float32)
    albedo = np.array([0.3, 0.7, 0.9], np.float32)
    tri_mat = (np.arange(f.shape[0]) % 3).astype(np.uint32)
    seed = 31
    engine.set_integrator(pt_bounces=4, albedo=0.7, seed=seed)
    engine.setLights((0.4, 0.4, 1.0), (0.2, 0, 0), (0, 0.2, 0), 20.0)
    plain = engine.renderFrame(None, 0, RENDER_PATH)
    engine.set_normals(vn, f)
    engine.set_materials(albedo, tri_mat)
    fb = engine.renderFrame(None, 0, RENDER_PATH)
    b.set_shading(vn, f, albedo, tri_mat)
    eps = float(np.float32(1e-4) * b.diag())
    img, _ = oracle.render_pt(b, ocam(oracle, cam), oracle.make_light(), 4, 0.7, eps, seed)
    assert np.array_equal(fb[:, 0], img)
    assert not np.array_equal(fb, plain)
    engine.set_normals(None)
    engine.set_materials(None)
    assert np.array_equal(engine.renderFrame(None, 0, RENDER_PATH), plain)
    from happyray_b200 import HRError
    with pytest.raises(HRError):
        engine.set_materials(albedo, np.full(f.shape[0], 3, np.uint32))   # index out of the table


@pytest.mark.parametrize("kind", [GRID_UNIFORM, GRID_TWO_LEVEL])
def test_render_primary_mode0(engine, oracle, c1_scene, kind):
    """Render mode 0 bit-exact against the oracle's simpleShade (SimpleIntegrator.h:41-126)
    over six progressive images: 0-3 take the 2 x 2 regular in-pixel pattern, 4 and 5 the
    Gaussian pixel sampler (RTEngine.cu:409-424)."""
    v, f = c1_scene
    gpu_build(engine, v, f, kind)
    b = oracle_build(oracle, v, f, kind)
    cam = S.camera_c1((64, 48))
    set_cam(engine, cam)
    seed = 777
    engine.set_integrator(seed=seed)
    fb, want = None, None
    for im in range(6):
        fb = engine.renderFrame(fb, im, RENDER_PRIMARY)
        want = oracle.render_primary(b, ocam(oracle, cam), im, seed, want)
        assert np.array_equal(fb, want), f"image {im}"
    miss = np.all(want == np.array([0.15, 0.2, 0.3], np.float32), axis=1)
    assert 0 < miss.sum() < miss.size


def test_render_rays_ray_file_mode(engine, oracle, small_clusters):
    """The ray-file form of render mode 0 (hr_render_rays_device): ray i traced and shaded by
    simpleShade into pixel i, bit-exact against the oracle, over two progressive images."""
    import torch
    v, f = small_clusters
    gpu_build(engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    rng = np.random.default_rng(12)
    n = 4000
    org = rng.uniform(v.min(0), v.max(0), (n, 3)).astype(np.float32)
    dirs = rng.normal(size=(n, 3)).astype(np.float32)
    d_org, d_dir = torch.from_numpy(org).cuda(), torch.from_numpy(dirs).cuda()
    d_fb = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    want = None
    for im in range(2):
        engine.render_rays_device(d_org, d_dir, n, im, d_fb)
        engine.sync()
        want = oracle.render_rays(b, org, dirs, im, want)
        assert np.array_equal(d_fb.cpu().numpy(), want)
    assert 0 < (want[:, 0] == 0.15).sum() < n


def test_radix_sort_and_scan_device(engine):
    import torch
    rng = np.random.default_rng(7)
    for n, bits in [(1, 1), (1000, 5), (123457, 17), (2_000_001, 24), (70000, 32)]:
        keys = rng.integers(0, 2 ** bits, n, dtype=np.uint64).astype(np.uint32)
        vals = np.arange(n, dtype=np.uint32)
        tk = torch.from_numpy(keys.view(np.int32)).cuda()
        tv = torch.from_numpy(vals.view(np.int32)).cuda()
        torch.cuda.synchronize()
        engine.radix_sort_pairs_device(tk, tv, n, bits)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(tk.cpu().numpy().view(np.uint32), keys[order])
        assert np.array_equal(tv.cpu().numpy().view(np.uint32), vals[order])
    for n in [1, 2047, 2048, 2049, 1_000_003]:
        x = rng.integers(0, 100, n).astype(np.uint32)
        tx = torch.from_numpy(x.view(np.int32)).cuda()
        torch.cuda.synchronize()
        engine.exclusive_scan_device(tx, n)
        want = np.concatenate([[0], np.cumsum(x, dtype=np.uint64)[:-1]]).astype(np.uint32)
        assert np.array_equal(tx.cpu().numpy().view(np.uint32), want)


def test_edge_cases(engine, oracle):
    # single triangle
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    f = np.array([[0, 1, 2]], np.uint32)
    for kind in (GRID_UNIFORM, GRID_TWO_LEVEL):
        gpu = gpu_build(engine, v, f, kind)
        assert_same_grid(gpu, oracle_build(oracle, v, f, kind))
        hid, t, u, vv = engine.trace_rays(np.array([[0.25, 0.25, 1.0]], np.float32), np.array([[0, 0, -1.0]], np.float32))
        assert hid[0] == 0 and abs(t[0] - 1) < 1e-6
    # a few huge overlapping triangles: pair counts far above the initial capacity estimate,
    # the build regrows from the device-computed totals and rebuilds
    rng = np.random.default_rng(3)
    v = rng.uniform(0, 1, (300, 3)).astype(np.float32)
    f = rng.integers(0, 300, (100, 3)).astype(np.uint32)
    for kind in (GRID_UNIFORM, GRID_TWO_LEVEL):
        gpu = gpu_build(engine, v, f, kind)
        b = oracle_build(oracle, v, f, kind)
        assert b.npairs > 6 * 100
        assert_same_grid(gpu, b)
    # degenerate triangles only
    v = np.array([[0, 0, 0], [1, 1, 1], [2, 2, 2]], np.float32)
    f = np.array([[0, 1, 2], [0, 0, 0]], np.uint32)
    gpu = gpu_build(engine, v, f, GRID_UNIFORM)
    assert_same_grid(gpu, oracle_build(oracle, v, f, GRID_UNIFORM))
    hid, *_ = engine.trace_rays(np.array([[0.5, 0.5, 3.0]], np.float32), np.array([[0, 0, -1.0]], np.float32))
    assert hid[0] == -1


@pytest.mark.parametrize("kind", [GRID_UNIFORM, GRID_TWO_LEVEL])
def test_axis_parallel_and_cell_boundary_rays(engine, oracle, small_clusters, kind):
    """Rays with zero direction components (infinite reciprocals), origins exactly on cell
    planes, origins outside the grid and rays grazing the grid box: ids, t, u, v equal to
    the oracle's, bit for bit."""
    v, f = small_clusters
    gpu_build(engine, v, f, kind)
    b = oracle_build(oracle, v, f, kind)
    gi = engine.grid_info()
    lo, hi, cs = (np.asarray(gi[k], np.float32) for k in ("bounds_min", "bounds_max", "cell_size"))
    rng = np.random.default_rng(11)
    dirs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
            (1, 1, 0), (0, -1, 1), (1, 0, -1), (1, 1, 1), (-1, 1, -1)]
    org, d = [], []
    for dv in dirs:
        dv = np.asarray(dv, np.float32) / np.float32(np.linalg.norm(dv))
        n = 400
        cells = rng.integers(0, np.asarray(gi["res"]), (n, 3))
        o = lo + cells.astype(np.float32) * cs                                 # cell corners
        o[: n // 2] += rng.uniform(0, 1, (n // 2, 3)).astype(np.float32) * cs  # ... and interiors
        o[n // 4: n // 2, 0] = lo[0] - 0.25                                    # outside the box
        o[-20:] = np.where(dv > 0, lo, np.where(dv < 0, hi, o[-20:]))          # on the box faces
        org.append(o.astype(np.float32))
        d.append(np.repeat(dv[None], n, 0))
    org, d = np.concatenate(org), np.concatenate(d)
    hid, t, u, vv = engine.trace_rays(org, d)
    ohid, ot, ou, ov = oracle.trace(b, org, d)
    assert np.array_equal(hid, ohid) and np.array_equal(t, ot)
    assert np.array_equal(u, ou) and np.array_equal(vv, ov)
    assert (hid >= 0).sum() > 100


def test_empty_mesh(engine):
    from happyray_b200 import HRError
    v = np.zeros((3, 3), np.float32)
    f = np.zeros((0, 3), np.uint32)
    engine.upload(v, v, f, 1.0)
    engine.build(GRID_TWO_LEVEL)
    hid, t, *_ = engine.trace_rays(np.zeros((2, 3), np.float32), np.array([[0, 0, 1.0], [1, 0, 0]], np.float32))
    assert np.all(hid == -1)
    with pytest.raises(HRError):
        engine.build(7)


# The product path against the reference's own kernels (tests/golden/ref_*.npz, made by
# tests/golden/make_ref_golden.py from the reference's build kernels and traversers).
GOLDEN = [p for p in sorted((Path(__file__).resolve().parent / "golden").glob("ref_*.npz")) if not p.name.startswith("ref_hier_")]


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
def test_gpu_matches_reference_golden(engine, path):
    from tests.test_oracle import cell_lists
    z = np.load(path)
    kind = int(z["kind"])
    dens, leaf = float(z["density"]), float(z["leaf_density"])
    gi, cells, leaves, prims = gpu_build(engine, z["vertices"], z["faces"], kind, bool(z["exact"]), ug=dens,
                                         top=dens, leaf=leaf if leaf > 0 else 2.0)
    assert gi["res"] == tuple(z["strict_res"])
    assert np.array_equal(gi["bounds_min"], z["strict_bmin"]) and np.array_equal(gi["cell_size_rcp"], z["strict_rcp"])
    if kind == GRID_UNIFORM:
        rc, rl = cell_lists(z["strict_cells"], z["strict_prims"])
        gc, gl = cell_lists(cells, prims)
    else:
        assert np.array_equal(cells, z["strict_cells"])
        rc, rl = cell_lists(z["strict_leaves"], z["strict_prims"])
        gc, gl = cell_lists(leaves, prims)
    assert np.array_equal(rc, gc) and np.array_equal(rl, gl)
    hid, t, _, _ = engine.trace_rays(z["ray_org"], z["ray_dir"])
    rid = z["strict_hit_id"].astype(np.int64)
    rid[rid == 0xFFFFFFFF] = -1
    assert np.array_equal(rid, hid)
    hit = hid >= 0
    assert np.all(np.abs(z["strict_hit_t"][hit] - t[hit]) <= 1e-5 * np.abs(t[hit]))


def test_scene_file_upload_renders_like_arrays(engine, tmp_path):
    """A scene.cfg key-frame sequence with camera and light, uploaded from files, renders
    the same AO and PT images as the same arrays given directly."""
    from tests.test_io import write_obj
    v, f = S.clusters(6_000, seed=4)
    frames = S.curl_keyframes(v, 3, amp=0.02, octaves=2, seed=4)
    for k in range(3):
        write_obj(tmp_path / ("fr%d.obj" % k), frames[k], f)
    cam = S.camera_at_bounds(v, (64, 48))
    (tmp_path / "camera.cfg").write_text(
        "position %r %r %r\norientation %r %r %r\nup 0 0 1\nresX 64\nresY 48\nFOV 60\n"
        % tuple(float(x) for x in list(cam["position"]) + list(cam["orientation"])))
    # a ceiling light: without its normal line the light would face edge1 x edge2 = +z, away
    # from the scene (LightSourceLoader.cpp:90-93)
    (tmp_path / "light.cfg").write_text("position 0.4 0.4 1\nnormal 0 0 -1\nintensity 20 20 20\n"
                                        "edge1 0.2 0 0\nedge2 0 0.2 0\n")
    (tmp_path / "scene.cfg").write_text("frame prefix = fr\nframe suffix = .obj\nnumber of frames = 3\n"
                                        "camera = camera.cfg\nlight = light.cfg\n")
    assert engine.upload_scene(str(tmp_path / "scene.cfg")) == (64, 48)
    outs = []
    for use_files in (True, False):
        if not use_files:
            engine.set_keyframes(frames, f)
            engine.setCamera(cam["position"], cam["orientation"], (0, 0, 1), 60.0, 64, 48)
            engine.setLights((0.4, 0.4, 1.0), (0.2, 0, 0), (0, 0.2, 0), 20.0)
        engine.set_frame_time(1.25, 0.0)
        engine.setGridDensities(0.0625, 2.0)
        engine.build(GRID_TWO_LEVEL)
        engine.set_integrator(ao_samples=4, ao_radius=-0.1, seed=3)
        outs.append((engine.renderFrame(None, 0, RENDER_AO), engine.renderFrame(None, 0, RENDER_PATH)))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_obj_normals_materials_upload_like_arrays(engine, tmp_path):
    """An OBJ with vn, usemtl and a .mtl, uploaded from the file, path-traces the same image
    as its arrays given through set_normals / set_materials; a plain OBJ uploaded after it
    drops them again."""
    from happyray_b200 import sceneio
    from tests.test_io import write_obj
    v, f = S.clusters(6_000, seed=8)
    rng = np.random.default_rng(8)
    vn = rng.normal(size=v.shape).astype(np.float32)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    (tmp_path / "m.mtl").write_text("newmtl a\nKd 0.2 0.3 0.4\nnewmtl b\nKd 0.9 0.9 0.6\n")
    with open(tmp_path / "s.obj", "w") as fh:
        fh.write("mtllib m.mtl\n")
        fh.writelines("v %.9g %.9g %.9g\n" % tuple(p) for p in v)
        fh.writelines("vn %.9g %.9g %.9g\n" % tuple(p) for p in vn)
        for i, t in enumerate(f):
            if i % 500 == 0:
                fh.write("usemtl %s\n" % "ab"[(i // 500) % 2])
            fh.write("f %d//%d %d//%d %d//%d\n" % (t[0] + 1, t[0] + 1, t[1] + 1, t[1] + 1, t[2] + 1, t[2] + 1))
    sc = sceneio.load_obj(str(tmp_path / "s.obj"))
    cam = S.camera_at_bounds(v, (64, 48))

    def frame():
        engine.set_frame_time(0.0, 0.0)
        engine.setGridDensities(0.0625, 2.0)
        engine.build(GRID_TWO_LEVEL)
        engine.setCamera(cam["position"], cam["orientation"], cam["up"], cam["fov"], 64, 48)
        engine.setLights((0.4, 0.4, 1.0), (0.2, 0, 0), (0, 0.2, 0), 20.0)
        engine.set_integrator(pt_bounces=3, albedo=0.7, seed=12)
        return engine.renderFrame(None, 0, RENDER_PATH)

    engine.upload_scene(str(tmp_path / "s.obj"))
    from_file = frame()
    engine.set_keyframes(sc.keyframes, sc.faces)
    engine.set_normals(sc.normals, sc.normal_idx)
    engine.set_materials(sc.albedo, sc.materials)
    assert np.array_equal(from_file, frame())
    write_obj(tmp_path / "plain.obj", v, f)
    engine.upload_scene(str(tmp_path / "plain.obj"))
    plain = frame()
    assert not np.array_equal(plain, from_file)
    engine.set_keyframes(sc.keyframes, sc.faces)
    assert np.array_equal(plain, frame())


def test_ray_query_files(engine, oracle, small_clusters, tmp_path):
    """.rays in, hits out: the ids and t of the oracle's closest hits."""
    from happyray_b200 import sceneio
    v, f = small_clusters
    gpu_build(engine, v, f, GRID_TWO_LEVEL)
    b = oracle_build(oracle, v, f, GRID_TWO_LEVEL)
    cam = S.camera_at_bounds(v, (40, 30))
    org, d = oracle.primary_rays(ocam(oracle, cam))
    sceneio.write_rays(str(tmp_path / "q.rays"), org, d)
    assert engine.trace_rays_file(str(tmp_path / "q.rays"), str(tmp_path / "q.hits")) == org.shape[0]
    rec = np.fromfile(tmp_path / "q.hits", dtype=[("id", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
    hid, t, u, vv = oracle.trace(b, org, d)
    assert np.array_equal(rec["id"], hid) and np.array_equal(rec["t"], t) and np.array_equal(rec["u"], u)
