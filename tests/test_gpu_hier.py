"""Instanced two-level grid hierarchy on the GPU (hr_hier_*): the object grids, the
instance grid and every hit must be bit-identical to the oracle's restatement of
TLGridHierarchySortBuilder.cu / TLGridHierarchyTraverser.h on the same inputs."""
import numpy as np
import pytest

from happyray_b200 import HRError
from happyray_b200 import scenes as S
from happyray_b200.hier import Hierarchy

pytestmark = pytest.mark.gpu


def rays(inst, n, seed, spread=0.03):
    rng = np.random.default_rng(seed)
    c = 0.5 * (inst["bmin"] + inst["bmax"])
    tgt = c[rng.integers(0, len(inst), n)] + rng.normal(0, spread, (n, 3))
    org = rng.uniform(-0.5, 1.5, (n, 3)).astype(np.float32)
    org[: n // 4] = tgt[: n // 4] + rng.normal(0, 0.002, (n // 4, 3))   # some rays start inside instances
    d = (tgt - org).astype(np.float32)
    d[: n // 4] = rng.normal(size=(n // 4, 3)).astype(np.float32)
    return org, d


def assert_same_build(h, ob):
    objs, oc, tri, tc, ii = h.download()
    for k in range(len(objs)):
        o = ob.objs[k]
        for f, g in (("bmin", "bmin"), ("bmax", "bmax"), ("cs", "cs"), ("rcp", "rcp"), ("res", "res")):
            assert np.array_equal(objs[f][k], np.array(list(getattr(o, g)), objs[f].dtype)), (k, f)
        assert (objs["cell_off"][k], objs["tri_begin"][k], objs["tri_count"][k]) == (o.cell_off, o.tri_begin, o.tri_count)
    assert np.array_equal(oc, ob.obj_cells)
    assert np.array_equal(tri, ob.prims)
    info = h.info()
    assert info["top_res"] == list(ob.top.res)
    assert np.array_equal(np.float32(info["top_bmin"]), np.array(list(ob.top.bmin), np.float32))
    assert np.array_equal(tc, ob.top_cells)
    assert np.array_equal(ii, ob.inst_ids)


def check_hits(h, ob, oracle, org, d):
    got = h.trace_rays(org, d)
    want = oracle.hier_trace(ob, org, d)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    # the same query into caller arrays (filled in place, returned as given)
    n = org.shape[0]
    out = [np.full(n, 7, np.int32), np.full(n, 7, np.int32)] + [np.full(n, 7.0, np.float32) for _ in range(3)]
    again = h.trace_rays(org, d, out=out)
    for a, o, g in zip(again, out, got):
        assert a is o and np.array_equal(a, g)
    return got


@pytest.mark.parametrize("seed,n_obj,n_inst,dens", [(1, 8, 300, (1.2, 1.2)), (2, 3, 40, (0.5, 3.0)),
                                                    (5, 16, 2000, (1.2, 1.2))])
def test_hier_build_and_trace_bitexact(hrlib, oracle, seed, n_obj, n_inst, dens):
    v, f, counts, inst = S.instanced_scene(n_obj, n_inst, seed=seed, tri_range=(80, 6000))
    ob = oracle.hier_build(v, f, counts, inst, *dens)
    with Hierarchy(0) as h:
        h.set_objects(v, f, counts)
        h.set_instances(inst)
        h.set_densities(*dens)
        h.build()
        assert_same_build(h, ob)
        org, d = rays(inst, 20000, seed + 10)
        hid, tid, t, u, vv = check_hits(h, ob, oracle, org, d)
        assert (hid >= 0).sum() > 2000
        # any hit below / beyond the closest t
        hit = hid >= 0
        occ_lo = h.occluded(org[hit], d[hit], t[hit] * np.float32(0.999))
        occ_hi = h.occluded(org[hit], d[hit], t[hit] * np.float32(1.001))
        w_lo = oracle.hier_trace(ob, org[hit], d[hit], tmax=t[hit] * np.float32(0.999), anyhit=True)[0] >= 0
        w_hi = oracle.hier_trace(ob, org[hit], d[hit], tmax=t[hit] * np.float32(1.001), anyhit=True)[0] >= 0
        assert np.array_equal(occ_lo, w_lo) and np.array_equal(occ_hi, w_hi)
        assert not occ_lo.any() and occ_hi.all()


def test_hier_rigid_frames_rebuild_the_instance_grid(hrlib, oracle):
    """A rigid-body animation: the instances move, the object grids stay."""
    v, f, counts, inst = S.instanced_scene(6, 500, seed=9, tri_range=(80, 3000))
    rng = np.random.default_rng(1)
    with Hierarchy(0) as h:
        h.set_objects(v, f, counts)
        for frame in range(3):
            moved = inst.copy()
            shift = rng.normal(0, 0.05, (len(inst), 3)).astype(np.float32) * frame
            moved["bmin"] += shift
            moved["bmax"] += shift
            # the world -> object translation moves opposite to the instance: x' = A (x - s) + b
            A = moved["m"].reshape(-1, 3, 4)[:, :, :3].astype(np.float64)
            mm = moved["m"].reshape(-1, 3, 4).astype(np.float64)
            mm[:, :, 3] -= np.einsum("nij,nj->ni", A, shift.astype(np.float64))
            moved["m"] = mm.reshape(-1, 12).astype(np.float32)
            h.set_instances(moved)
            h.build()
            ob = oracle.hier_build(v, f, counts, moved, 1.2, 1.2)
            assert_same_build(h, ob)
            org, d = rays(moved, 5000, 30 + frame)
            check_hits(h, ob, oracle, org, d)


def test_hier_single_instance_and_misses(hrlib, oracle):
    v, f = S.icosphere(4)
    v = np.asarray(v, np.float32)
    counts = np.array([len(f)], np.uint32)
    inst = np.zeros(1, S.INSTANCE_DTYPE)
    inst[0] = S.instance_record(0, np.concatenate([np.eye(3) * 0.5, [[0.2], [0.3], [0.4]]], axis=1),
                                v.min(0), v.max(0))
    ob = oracle.hier_build(v, f, counts, inst, 1.2, 1.2)
    with Hierarchy(0) as h:
        h.set_objects(v, f, counts)
        h.set_instances(inst)
        h.build()
        assert_same_build(h, ob)
        org, d = rays(inst, 4000, 3, spread=0.4)
        check_hits(h, ob, oracle, org, d)
        # rays pointing away from everything
        far = np.full((100, 3), 50.0, np.float32)
        hid, tid, t, _, _ = h.trace_rays(far, np.ones((100, 3), np.float32))
        assert np.all(hid == -1) and np.all(tid == -1) and np.all(t == np.float32(3.4028235e38))


def test_hier_rejects_bad_input(hrlib):
    v, f = S.icosphere(2)
    v = np.asarray(v, np.float32)
    with Hierarchy(0) as h:
        with pytest.raises(HRError):
            h.set_objects(v, f, [len(f) - 1])            # counts do not sum to the triangles
        with pytest.raises(HRError):
            h.set_objects(v, f, [len(f), 0])             # an empty object
        bad = np.asarray(f).copy()
        bad[0, 0] = v.shape[0]
        with pytest.raises(HRError):
            h.set_objects(v, bad, [len(f)])
        with pytest.raises(HRError):
            h.build()                                     # nothing set
        h.set_objects(v, f, [len(f)])
        inst = np.zeros(1, S.INSTANCE_DTYPE)
        inst[0] = S.instance_record(0, np.concatenate([np.eye(3), np.zeros((3, 1))], axis=1), v.min(0), v.max(0))
        wrong = inst.copy()
        wrong["obj"] = 1
        with pytest.raises(HRError):
            h.set_instances(wrong)
        with pytest.raises(HRError):
            h.trace_rays(np.zeros((1, 3), np.float32), np.ones((1, 3), np.float32))   # not built
        h.set_instances(inst)
        h.build()
        hid, _, _, _, _ = h.trace_rays(np.array([[0, 0, -5]], np.float32), np.array([[0, 0, 1]], np.float32))
        assert hid[0] == 0


HIER_GOLDEN = sorted((__import__("pathlib").Path(__file__).resolve().parent / "golden").glob("ref_hier_*.npz"))


@pytest.mark.parametrize("path", HIER_GOLDEN, ids=lambda p: p.stem)
def test_gpu_hier_matches_reference_golden(hrlib, path):
    """The GPU hierarchy against the reference's own builder and traverser (fixtures of
    tests/golden/make_ref_golden.py --hier, IEEE build): the same instance grid, object
    grid parameters, and the same instance and triangle for every ray."""
    z = np.load(path)
    with Hierarchy(0) as h:
        h.set_objects(z["vertices"], z["faces"], z["counts"])
        h.set_instances(z["instances"])
        h.set_densities(float(z["top_density"]), float(z["object_density"]))
        h.build()
        objs, _, _, tc, ii = h.download()
        assert np.array_equal(objs["res"], z["strict_obj_res"])
        assert np.array_equal(objs["cell_off"], z["strict_obj_first"])
        info = h.info()
        assert info["top_res"] == list(z["strict_top_res"])
        # per-cell instance lists (the reference's in-cell order comes from its sort of
        # keys only, so compare each list sorted)
        rc = z["strict_top_cells"]
        for c in range(rc.shape[0]):
            assert np.array_equal(np.sort(z["strict_inst_ids"][rc[c, 0]:rc[c, 1]]), np.sort(ii[tc[c, 0]:tc[c, 1]]))
        hid, tid, t, _, _ = h.trace_rays(z["ray_org"], z["ray_dir"])
    ri = z["strict_hit_inst"].astype(np.int64)
    ri[ri == 0xFFFFFFFF] = -1
    rt = z["strict_hit_tri"].astype(np.int64)
    rt[rt == 0xFFFFFFFF] = -1
    assert np.array_equal(ri, hid) and np.array_equal(rt, tid)
    hit = hid >= 0
    rel = np.abs(z["strict_hit_t"][hit] - t[hit]) / np.abs(t[hit])
    assert rel.max() <= 5e-6
