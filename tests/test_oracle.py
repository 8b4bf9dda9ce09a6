"""CPU tests of the oracle: known answers, independent restatements and the invariants the
reference keeps as commented-out debug checks (UGridSortBuilder.h:253-399,
TLGridSortBuilder.h:411-428)."""
import math
from pathlib import Path

import numpy as np
import pytest

from conftest import as_v4


def f32(x):
    return np.float32(x)


# -- known answers -----------------------------------------------------------------------

def test_pcg32_known_answer(oracle):
    # pcg32-demo (O'Neill, pcg-c-basic): pcg32_srandom_r(&rng, 42u, 54u) -> first outputs
    expect_u32 = [0xA15C02B7, 0x7B47F409, 0xBA1D3330, 0x83D2F293, 0xBFA4784B, 0xCBED606E]
    got = oracle.pcg32_floats(42, 54, 6)
    want = np.array([(x >> 8) * 2.0 ** -24 for x in expect_u32], np.float32)
    assert np.array_equal(got, want)


def test_sincos2pi_accuracy(oracle):
    us = np.linspace(0.0, 1.0, 20001, endpoint=False, dtype=np.float32)
    err = 0.0
    for u in us[::7]:
        s, c = oracle.sincos2pi(float(u))
        err = max(err, abs(s - math.sin(2 * math.pi * float(u))), abs(c - math.cos(2 * math.pi * float(u))))
    assert err < 5e-7


def test_log_series_accuracy(oracle):
    """The Gaussian pixel sampler's logarithm (atanh series) against math.log over the
    range it is used on, 1 - u for u in [0, 1): absolute error below 1e-6."""
    xs = np.concatenate([np.float32(2.0) ** -np.arange(0, 25),
                         np.random.default_rng(5).uniform(2.0 ** -24, 1.0, 4000).astype(np.float32)])
    err = max(abs(oracle.log_series(float(x)) - math.log(float(x))) for x in xs)
    assert err < 1e-6


def test_pow_third_close_to_cube_root(oracle):
    for x in [1e-6, 0.37, 1.0, 27.0, 1234.5, 5.0 * 32768 / 0.2, 3.3e7]:
        y = oracle.pow_third(x)
        # x ** 0.3333333f, the reference's exponent (UGridSortBuilder.h:83)
        ref = float(np.float32(float(x) ** float(np.float32(0.3333333))))
        assert y == ref


def test_lerp_bounds_matches_numpy(oracle, small_clusters):
    v, _ = small_clusters
    rng = np.random.default_rng(5)
    v2 = (v + rng.normal(0, 0.01, v.shape)).astype(np.float32)
    c = f32(0.37)
    out, bmin, bmax = oracle.lerp_bounds(v, v2, float(c))
    want = v * (f32(1) - c) + v2 * c    # float32 numpy: same operation order, no FMA
    assert np.array_equal(out[:, :3], want)
    assert np.all(out[:, 3] == 0)
    lo, hi = want.min(0), want.max(0)
    d = hi - lo
    diag = np.sqrt(f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
    pad = f32(0.001) * diag
    assert np.array_equal(bmin, lo - pad) and np.array_equal(bmax, hi + pad)


# -- uniform grid -------------------------------------------------------------------------

def bbox_cells_numpy(v4, idx, g):
    """Independent numpy restatement of the bounding-box cell range (UniformGridBuildKernels.h:56-73)."""
    p = v4[idx][:, :, :3]
    lo, hi = p.min(1), p.max(1)
    bmin = np.array(g.bmin, np.float32)
    rcp = np.array(g.rcp, np.float32)
    res = np.array(g.res, np.int64)
    a = ((lo - bmin) * rcp)
    b = ((hi - bmin) * rcp + f32(1.0))
    clo = np.maximum(0, np.trunc(a).astype(np.int64))
    chi = np.minimum(res, np.trunc(b).astype(np.int64))
    return clo, chi


def check_ranges(cells, prims, ncells, npairs, ntri, valid_end=None):
    assert cells.shape == (ncells, 2)
    b, e = cells[:, 0].astype(np.int64), cells[:, 1].astype(np.int64)
    assert np.all(b <= e) and np.all(e <= npairs)
    ne = e > b
    # non-empty ranges are disjoint and appear in cell order
    bb, ee = b[ne], e[ne]
    assert np.all(bb[1:] >= ee[:-1])
    assert np.all(prims < ntri)
    for cb, ce in zip(bb[:2000], ee[:2000]):
        seg = prims[cb:ce]
        assert np.all(np.diff(seg.astype(np.int64)) > 0), "cell list must be strictly ascending"
    return ne


@pytest.mark.parametrize("exact", [False, True])
def test_ug_build_c1(oracle, c1_scene, exact):
    v, f = c1_scene
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    b = oracle.build_ug(v4, f, bmin, bmax, 5.0, exact)
    assert b.res == (94, 94, 18)
    ne = check_ranges(b.cells, b.prims, b.grid.ncells, b.npairs, f.shape[0])
    clo, chi = bbox_cells_numpy(v4, f, b.grid)
    counts = np.prod(np.maximum(chi - clo, 0), axis=1)
    assert b.npairs == counts.sum()
    # every reference of a cell lies in that cell's bbox range; bbox insertion covers all of them
    res = b.res
    tri_sets = {}
    cell_ids = np.nonzero(ne)[0]
    for c in cell_ids[::37]:
        x, y, z = c % res[0], (c // res[0]) % res[1], c // (res[0] * res[1])
        ins = (clo[:, 0] <= x) & (x < chi[:, 0]) & (clo[:, 1] <= y) & (y < chi[:, 1]) & (clo[:, 2] <= z) & (z < chi[:, 2])
        want = np.nonzero(ins)[0]
        got = b.prims[b.cells[c, 0]:b.cells[c, 1]]
        if exact:
            assert set(got.tolist()) <= set(want.tolist())
        else:
            assert np.array_equal(got, want)
        tri_sets[c] = got
    if not exact:
        assert (b.cells[:, 1] - b.cells[:, 0]).sum() == b.npairs


def _sat_ref_f64(tri, c, h, eps):
    """The reference's triangle/box test (UniformGridBuildKernels.cu:8-48, 323-366) in double:
    plane test plus the 9 edge-cross axes, unnormalised axes with absolute slack `eps`."""
    v = tri - c
    e = [v[1] - v[0], v[2] - v[1], v[0] - v[2]]
    n = np.cross(v[1] - v[0], v[2] - v[0])
    vmin = np.where(n > 0, -h, h) - v[0]
    vmax = np.where(n > 0, h, -h) - v[0]
    if not (n @ vmin <= 0 and n @ vmax > 0):
        return False
    for j in range(3):
        for i in range(3):
            a = np.cross(e[j], np.eye(3)[i])
            p = v @ a
            r = np.abs(a) @ h
            if p.min() > r + eps or p.max() + eps < -r:
                return False
    return True


def test_ug_exact_sat_property(oracle, c1_scene):
    """Exact insertion keeps a bbox cell iff the reference's triangle/box test passes: a kept
    cell passes the double-precision test with slightly looser bounds, a dropped cell fails it
    with slightly tighter bounds (half size 0.505 cell, slack 1e-5)."""
    v, f = c1_scene
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    bx = oracle.build_ug(v4, f, bmin, bmax, 5.0, False)
    be = oracle.build_ug(v4, f, bmin, bmax, 5.0, True)
    g = be.grid
    cs = np.array(g.cs, np.float64)
    b0 = np.array(g.bmin, np.float64)
    res = be.res
    rng = np.random.default_rng(0)
    cells = np.nonzero(bx.cells[:, 1] > bx.cells[:, 0])[0]
    checked = dropped = 0
    for c in rng.choice(cells, 400, replace=False):
        allt = set(bx.prims[bx.cells[c, 0]:bx.cells[c, 1]].tolist())
        acc = set(be.prims[be.cells[c, 0]:be.cells[c, 1]].tolist())
        assert acc <= allt
        x, y, z = c % res[0], (c // res[0]) % res[1], c // (res[0] * res[1])
        # the reference centres its test box at min corner + 0.505 cell (UniformGridBuildKernels.cu:275-281)
        centre = b0 + np.array([x, y, z]) * cs + 0.505 * cs
        for t in allt:
            tri = v4[f[t], :3].astype(np.float64)
            if t in acc:
                assert _sat_ref_f64(tri, centre, 0.506 * cs, 1.01e-5)
            else:
                assert not _sat_ref_f64(tri, centre, 0.504 * cs, 0.99e-5)
                dropped += 1
            checked += 1
    assert checked > 400 and dropped > 0


# -- two-level grid -------------------------------------------------------------------------

def test_tl_build_invariants(oracle, small_clusters):
    v, f = small_clusters
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    b = oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)
    C = b.grid.ncells
    assert b.cells.shape == (C, 2)
    y = b.cells[:, 1]
    rx, ry, rz = y & 0xFF, (y >> 8) & 0xFF, (y >> 16) & 0xFF
    assert np.all(rx >= 1) and np.all(ry >= 1) and np.all(rz >= 1)
    is_leaf = (y & 0x10000000) != 0
    not_empty = (y & 0x40000000) != 0
    # leaf flag => 1x1x1 sub-grid
    assert np.all((rx[is_leaf] == 1) & (ry[is_leaf] == 1) & (rz[is_leaf] == 1))
    # leaf ranges are allocated contiguously in top-cell order (prepareTopLevelCellRanges)
    nl = (rx * ry * rz).astype(np.int64)
    assert np.array_equal(b.cells[:, 0].astype(np.int64), np.concatenate([[0], np.cumsum(nl)[:-1]]))
    assert nl.sum() == b.leaves.shape[0]
    # leaves: valid ranges, disjoint, ascending ids
    check_ranges(b.leaves, b.prims, b.leaves.shape[0], b.npairs, f.shape[0])
    # empty top cells have only empty leaves
    for c in np.nonzero(~not_empty)[0][:500]:
        s = b.cells[c, 0]
        assert np.all(b.leaves[s:s + nl[c]] == 0)
    assert (b.leaves[:, 1] - b.leaves[:, 0]).sum() == b.npairs


# -- traversal --------------------------------------------------------------------------------

def compare_fp64(oracle, v4, f, org, d, hid, t, u, v, tol=1e-5):
    """Ids equal to the FP64 brute force except at flagged ties / edges / grazing hits;
    t and the barycentric weights u, v within `tol` relative; and the hit point from (u, v)
    within `tol` relative to its magnitude."""
    bid, bt, bu, bv, fl = oracle.brute_f64(v4, f, org, d)
    unflagged = fl == 0
    assert np.array_equal(hid[unflagged], bid[unflagged])
    m = unflagged & (bid >= 0)
    assert np.all(np.abs(t[m] - bt[m]) <= tol * bt[m])
    assert np.all(np.abs(u[m] - bu[m]) <= tol * np.abs(bu[m]) + 1e-30)
    assert np.all(np.abs(v[m] - bv[m]) <= tol * np.abs(bv[m]) + 1e-30)
    tri = v4[f[bid[m]]][:, :, :3].astype(np.float64)
    e1, e2 = tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]
    dp = (u[m] - bu[m])[:, None] * e1 + (v[m] - bv[m])[:, None] * e2
    pmag = np.linalg.norm(tri[:, 0] + bu[m][:, None] * e1 + bv[m][:, None] * e2, axis=1) + bt[m]
    assert np.all(np.linalg.norm(dp, axis=1) <= tol * pmag)
    return unflagged.mean(), m.sum()


@pytest.mark.parametrize("kind", ["ug", "tl"])
def test_trace_matches_fp64_c1(oracle, c1_scene, kind):
    from happyray_b200 import scenes as S
    v, f = c1_scene
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    b = oracle.build_ug(v4, f, bmin, bmax, 5.0, True) if kind == "ug" else oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)
    cam = S.camera_c1()
    oc = oracle.camera(cam["position"], cam["orientation"], cam["up"], cam["fov"], 256, 256)
    org, d = oracle.primary_rays(oc)
    hid, t, u, vv = oracle.trace_primary(b, oc)
    sel = np.random.default_rng(1).choice(org.shape[0], 3000, replace=False)
    frac, nhit = compare_fp64(oracle, v4, f, org[sel], d[sel], hid[sel], t[sel], u[sel], vv[sel])
    assert frac > 0.99 and nhit > 300
    # random rays from inside the scene in all directions
    rng = np.random.default_rng(2)
    o2 = rng.uniform([0, 0, -0.05], [1, 1, 0.15], (2000, 3)).astype(np.float32)
    d2 = rng.normal(size=(2000, 3)).astype(np.float32)
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    h2 = oracle.trace(b, o2, d2)
    frac, nhit = compare_fp64(oracle, v4, f, o2, d2, *h2)
    assert frac > 0.98 and nhit > 500


def test_ug_tl_agree(oracle, small_clusters):
    """Uniform and two-level grids over the same scene give the same closest hits."""
    from happyray_b200 import scenes as S
    v, f = small_clusters
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    bu = oracle.build_ug(v4, f, bmin, bmax, 5.0, True)
    bt = oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)
    cam = S.camera_at_bounds(v, (96, 96))
    oc = oracle.camera(cam["position"], cam["orientation"], cam["up"], cam["fov"], 96, 96)
    h1 = oracle.trace_primary(bu, oc)
    h2 = oracle.trace_primary(bt, oc)
    org, d = oracle.primary_rays(oc)
    _, _, _, _, fl = oracle.brute_f64(v4, f, org, d)
    ok = fl == 0
    assert np.array_equal(h1[0][ok], h2[0][ok])
    assert np.array_equal(h1[1][ok], h2[1][ok])


def test_ao_pt_sanity(oracle, small_clusters):
    from happyray_b200 import scenes as S
    v, f = small_clusters
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    b = oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)
    cam = S.camera_at_bounds(v, (64, 48))
    oc = oracle.camera(cam["position"], cam["orientation"], cam["up"], cam["fov"], 64, 48)
    alpha = float(np.float32(0.1) * b.diag())
    img, rays = oracle.render_ao(b, oc, 8, alpha, 7)
    hid, *_ = oracle.trace_primary(b, oc)
    assert np.all((img >= 0) & (img <= 1))
    assert np.all(img[hid < 0] == 1.0)
    assert rays == 64 * 48 + 8 * int((hid >= 0).sum())
    img2, _ = oracle.render_ao(b, oc, 8, alpha, 7)
    assert np.array_equal(img, img2)
    light = oracle.make_light()
    pt, prays = oracle.render_pt(b, oc, light, 4, 0.7, float(np.float32(1e-4) * b.diag()), 11)
    assert np.all(np.isfinite(pt)) and np.all(pt >= 0) and pt.max() > 0
    assert prays >= 64 * 48


def test_edge_cases(oracle):
    # empty mesh: every ray misses
    v = np.zeros((0, 3), np.float32)
    f = np.zeros((0, 3), np.uint32)
    v4 = as_v4(np.array([[0, 0, 0], [1, 1, 1]], np.float32))
    b = oracle.build_ug(v4, f, np.zeros(3, np.float32), np.ones(3, np.float32), 5.0, True)
    assert b.npairs == 0
    hid, t, u, vv = oracle.trace(b, np.zeros((4, 3), np.float32), np.tile([0.0, 0.0, 1.0], (4, 1)).astype(np.float32))
    assert np.all(hid == -1)
    # single triangle, ray straight through its centroid
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    f = np.array([[0, 1, 2]], np.uint32)
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    for b in (oracle.build_ug(v4, f, bmin, bmax, 5.0, True), oracle.build_tl(v4, f, bmin, bmax, 0.0625, 2.0)):
        hid, t, u, vv = oracle.trace(b, np.array([[0.25, 0.25, 1.0]], np.float32), np.array([[0, 0, -1.0]], np.float32))
        assert hid[0] == 0 and abs(t[0] - 1.0) < 1e-6 and abs(u[0] - 0.25) < 1e-6 and abs(vv[0] - 0.25) < 1e-6
    # degenerate (zero-area) triangle is never hit
    v = np.array([[0, 0, 0], [1, 1, 1], [2, 2, 2], [0, 0, 1], [1, 0, 1], [0, 1, 1]], np.float32)
    f = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    v4, bmin, bmax = oracle.lerp_bounds(v, v, 1.0)
    b = oracle.build_ug(v4, f, bmin, bmax, 5.0, True)
    hid, *_ = oracle.trace(b, np.array([[0.2, 0.2, 3.0], [1.0, 1.0, 3.0]], np.float32),
                           np.array([[0, 0, -1.0], [0, 0, -1.0]], np.float32))
    assert hid[0] == 1 and hid[1] == -1


# ---------------------------------------------------------------------------------
# Pin against the reference itself: tests/golden/ref_*.npz hold what the reference's own
# build kernels and traversers computed on a B200 (tests/golden/make_ref_golden.py runs
# them through oracle/ref_pin), for an IEEE build of the reference (strict) and for its
# shipped -use_fast_math build (fast).

GOLDEN = [p for p in sorted((Path(__file__).resolve().parent / "golden").glob("ref_*.npz")) if not p.name.startswith("ref_hier_")]


def cell_lists(cells, prims):
    """(per-cell counts, the concatenated per-cell lists each sorted by triangle id): the
    reference's order inside a cell depends on atomics, the oracle's is ascending."""
    cells = np.asarray(cells, np.int64).reshape(-1, 2)
    cnt = np.where(cells[:, 1] > cells[:, 0], cells[:, 1] - cells[:, 0], 0)
    parts = [np.sort(prims[cells[c, 0]:cells[c, 1]]) for c in np.nonzero(cnt)[0]]
    return cnt, (np.concatenate(parts) if parts else np.zeros(0, np.uint32))


def oracle_for_golden(O, z):
    v, f = z["vertices"], z["faces"]
    v4, bmin, bmax = O.lerp_bounds(v, v, 1.0)
    if int(z["kind"]) == 0:
        return O.build_ug(v4, f, bmin, bmax, float(z["density"]), bool(z["exact"]))
    return O.build_tl(v4, f, bmin, bmax, float(z["density"]), float(z["leaf_density"]))


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
@pytest.mark.parametrize("variant", ["strict", "fast"])
def test_oracle_matches_reference_golden(oracle, path, variant):
    z = np.load(path)
    b = oracle_for_golden(oracle, z)
    g = b.grid

    def r(k):
        return z[f"{variant}_{k}"]

    # grid parameters: bit-exact
    assert tuple(r("res")) == tuple(g.res)
    for k in ("bmin", "bmax", "cs", "rcp"):
        assert np.array_equal(r(k), np.array(getattr(g, k), np.float32)), k
    # per-cell (uniform) or packed top cells + per-leaf (two-level) lists: exact
    if int(z["kind"]) == 0:
        rc, rl = cell_lists(r("cells"), r("prims"))
        oc, ol = cell_lists(b.cells, np.asarray(b.prims))
    else:
        assert np.array_equal(r("cells"), np.asarray(b.cells, np.uint32).reshape(-1, 2))
        rc, rl = cell_lists(r("leaves"), r("prims"))
        oc, ol = cell_lists(b.leaves, np.asarray(b.prims))
    assert np.array_equal(rc, oc)
    assert np.array_equal(rl, ol)
    # closest hits of the camera rays: ids equal, t within 1e-5 relative (the reference
    # re-derives the direction from its reciprocal with an approximate division)
    hid, t, _, _ = oracle.trace(b, z["ray_org"], z["ray_dir"])
    rid = r("hit_id").astype(np.int64)
    rid[rid == 0xFFFFFFFF] = -1
    assert np.array_equal(rid, hid)
    hit = hid >= 0
    assert hit.sum() > 500
    rel = np.abs(r("hit_t")[hit] - t[hit]) / np.abs(t[hit])
    assert rel.max() <= 1e-5
