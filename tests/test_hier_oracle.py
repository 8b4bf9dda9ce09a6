"""Instanced two-level grid hierarchy, CPU side: the oracle's object grids, instance grid
and nested traversal (TLGridHierarchySortBuilder.cu, TLGridHierarchyTraverser.h) checked
against their invariants and against an FP64 brute force over every instance."""
import numpy as np
import pytest

from happyray_b200 import scenes as S


def small_scene(seed=3):
    return S.instanced_scene(4, 48, seed=seed, tri_range=(80, 1500), world=1.0, scale_range=(0.08, 0.25))


def rays_at_instances(inst, n, seed):
    rng = np.random.default_rng(seed)
    c = 0.5 * (inst["bmin"] + inst["bmax"])
    tgt = c[rng.integers(0, len(inst), n)] + rng.normal(0, 0.03, (n, 3))
    org = rng.uniform(-0.5, 1.5, (n, 3)).astype(np.float32)
    d = (tgt - org).astype(np.float32)
    return org, d


def brute(v, f, counts, inst, org, dirs):
    """Closest accepted hit over all instances in FP64: the ray in object space, every
    triangle of the object, t inside the instance box interval.  Returns (inst, tri, t,
    second-best t)."""
    starts = np.concatenate([[0], np.cumsum(np.asarray(counts, np.int64))])
    n = org.shape[0]
    best_i = np.full(n, -1); best_tri = np.full(n, -1); best_t = np.full(n, np.inf); second = np.full(n, np.inf)
    o64, d64 = org.astype(np.float64), dirs.astype(np.float64)
    for ii, rec in enumerate(inst):
        M = rec["m"].astype(np.float64).reshape(3, 4)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = 1.0 / d64
            a = (rec["bmin"].astype(np.float64) - o64) * r
            b = (rec["bmax"].astype(np.float64) - o64) * r
            te = np.max(np.minimum(a, b), axis=1)
            tx = np.min(np.maximum(a, b), axis=1)
        ok = (tx > te) & (tx >= 0)
        if not ok.any():
            continue
        ot = o64 @ M[:, :3].T + M[:, 3]
        dt = d64 @ M[:, :3].T
        ob = int(rec["obj"])
        tri = f[starts[ob]:starts[ob + 1]]
        p0, p1, p2 = [v[tri[:, k]].astype(np.float64) for k in range(3)]
        e1, e2 = p1 - p0, p2 - p0
        for i in np.nonzero(ok)[0]:
            p = np.cross(dt[i], e2)
            det = np.einsum("ij,ij->i", e1, p)
            with np.errstate(divide="ignore", invalid="ignore"):
                inv = 1.0 / det
                sv = ot[i] - p0
                u = np.einsum("ij,ij->i", sv, p) * inv
                q = np.cross(sv, e1)
                vv = (q @ dt[i]) * inv
                t = np.einsum("ij,ij->i", e2, q) * inv
            hit = (u >= 0) & (vv >= 0) & (u + vv <= 1) & (t > 1e-4) & (t >= te[i]) & (t < tx[i])
            for k in np.nonzero(hit)[0]:
                if t[k] < best_t[i]:
                    second[i] = best_t[i]
                    best_t[i], best_i[i], best_tri[i] = t[k], ii, starts[ob] + k
                else:
                    second[i] = min(second[i], t[k])
    return best_i, best_tri, best_t, second


def test_oracle_hier_build_invariants(oracle):
    v, f, counts, inst = small_scene()
    h = oracle.hier_build(v, f, counts, inst, 1.2, 1.2)
    starts = np.concatenate([[0], np.cumsum(np.asarray(counts, np.int64))])
    total = 0
    for k in range(len(counts)):
        o = h.objs[k]
        assert (o.tri_begin, o.tri_count) == (starts[k], counts[k])
        assert o.cell_off == total
        total += o.res[0] * o.res[1] * o.res[2]
        cells = h.obj_cells[o.cell_off:total]
        lists = [h.prims[b:e] for b, e in cells]
        ids = np.concatenate(lists) if lists else np.zeros(0)
        # each cell's list is ascending and holds only the object's triangles; every triangle is listed
        assert all(np.all(np.diff(x) > 0) for x in lists)
        assert ids.min() >= starts[k] and ids.max() < starts[k + 1]
        assert np.array_equal(np.unique(ids), np.arange(starts[k], starts[k + 1]))
    assert h.obj_cells.shape[0] == total
    assert h.obj_cells[:, 1].max() == h.prims.shape[0]
    # instance grid: each cell ascending; every instance listed
    lists = [h.inst_ids[b:e] for b, e in h.top_cells]
    assert all(np.all(np.diff(x) > 0) for x in lists)
    assert np.array_equal(np.unique(h.inst_ids), np.arange(len(inst)))


def test_oracle_hier_trace_matches_brute_force(oracle):
    v, f, counts, inst = small_scene()
    h = oracle.hier_build(v, f, counts, inst, 1.2, 1.2)
    org, d = rays_at_instances(inst, 400, 7)
    hi, ht, t, u, vv = oracle.hier_trace(h, org, d)
    bi, bt, btt, second = brute(v, f, counts, inst, org, d)
    hits = bi >= 0
    assert hits.sum() > 150
    assert np.array_equal(hi >= 0, hits)
    clear = hits & (second > btt * (1 + 1e-4))
    assert clear.sum() > 100
    assert np.array_equal(hi[clear], bi[clear]) and np.array_equal(ht[clear], bt[clear])
    assert np.allclose(t[clear], btt[clear], rtol=1e-4)
    # any-hit below the closest t: never occluded; just beyond it: occluded
    ai, _, _, _, _ = oracle.hier_trace(h, org[hits], d[hits], tmax=t[hits] * (1 - 1e-3), anyhit=True)
    bi2, _, _, _, _ = oracle.hier_trace(h, org[hits], d[hits], tmax=t[hits] * (1 + 1e-3), anyhit=True)
    assert np.all(ai < 0) and np.all(bi2 >= 0)


def test_oracle_hier_identity_instances_equal_plain_objects(oracle):
    """One identity instance per object, objects disjoint: hits are the triangles'
    own hits, found through the object grids."""
    v, f = S.icosphere(3)
    v = np.asarray(v, np.float32) * 0.3
    v2 = v + np.float32(1.0)
    verts = np.concatenate([v, v2])
    faces = np.concatenate([f, np.asarray(f) + v.shape[0]]).astype(np.uint32)
    counts = np.array([len(f), len(f)], np.uint32)
    inst = np.zeros(2, S.INSTANCE_DTYPE)
    for k, vv in enumerate((v, v2)):
        inst[k] = S.instance_record(k, np.concatenate([np.eye(3), np.zeros((3, 1))], axis=1), vv.min(0), vv.max(0))
    h = oracle.hier_build(verts, faces, counts, inst, 1.2, 1.2)
    rng = np.random.default_rng(0)
    org = rng.uniform(-1, 2, (300, 3)).astype(np.float32)
    tgt = np.where(rng.random((300, 1)) < 0.5, 0.0, 1.0) + rng.normal(0, 0.1, (300, 3))
    d = (tgt - org).astype(np.float32)
    hi, ht, t, _, _ = oracle.hier_trace(h, org, d)
    bi, bt, btt, second = brute(verts, faces, counts, inst, org, d)
    clear = (bi >= 0) & (second > btt * (1 + 1e-4))
    assert clear.sum() > 100
    assert np.array_equal(ht[clear], bt[clear])
    assert np.array_equal(hi[clear], np.where(bt[clear] < len(f), 0, 1))


def test_instances_file_round_trip(hrlib, tmp_path):
    from happyray_b200 import hier as Hh
    from happyray_b200 import HRError
    import pytest
    _, _, _, inst = small_scene()
    p = tmp_path / "scene.instances"
    Hh.write_instances(str(p), inst)
    text = p.read_text()
    assert text.count("obj_id") == len(inst) and "m_row_2" in text and "AABB_max" in text
    back = Hh.read_instances(str(p))
    assert back.dtype == Hh.INSTANCE_DTYPE
    for k in ("obj", "m", "bmin", "bmax"):
        assert np.array_equal(back[k], inst[k])
    # the reference's reader: defaults for missing rows, comments, other keys ignored
    q = tmp_path / "b.instances"
    q.write_text("# header\nobj_id 3\nm_row_0 1 0 0 5 # translated\nfoo bar\nAABB_min 0 0 0\nAABB_max 1 1 1\n"
                 "obj_id 1\n")
    r = Hh.read_instances(str(q))
    assert list(r["obj"]) == [3, 1]
    assert np.array_equal(r["m"][0], [1, 0, 0, 5, 0, 1, 0, 0, 0, 0, 1, 0])
    assert np.array_equal(r["bmax"][0], [1, 1, 1])
    (tmp_path / "c.instances").write_text("m_row_0 1 0 0 0\n")
    with pytest.raises(HRError):
        Hh.read_instances(str(tmp_path / "c.instances"))


HIER_GOLDEN = sorted((__import__("pathlib").Path(__file__).resolve().parent / "golden").glob("ref_hier_*.npz"))


@pytest.mark.parametrize("path", HIER_GOLDEN, ids=lambda p: p.stem)
@pytest.mark.parametrize("variant", ["strict", "fast"])
def test_oracle_hier_matches_reference_golden(oracle, path, variant):
    """The oracle against the reference's own hierarchy builder and traverser
    (oracle/ref_pin/ref_pin_hier.cu, fixtures by tests/golden/make_ref_golden.py --hier).
    Everything is exact but the object-cell lists: the reference's UniformGrid recomputes
    each object grid's cell size and reciprocal with an approximate division on the device
    (fastDivide, UniformGrid.h:58-75), so a triangle lying exactly on a cell boundary can
    be binned one cell over; the oracle keeps the IEEE quotients RTEngine computes
    (RTEngine.cu:325-327).  Those triangles must still sit in the same cells up to one
    boundary layer, and every hit must agree."""
    from test_oracle import cell_lists
    z = np.load(path)
    ob = oracle.hier_build(z["vertices"], z["faces"], z["counts"], z["instances"], float(z["top_density"]),
                           float(z["object_density"]))

    def r(k):
        return z[f"{variant}_{k}"]

    for k in range(len(z["counts"])):
        o = ob.objs[k]
        assert tuple(r("obj_res")[k]) == tuple(o.res)
        assert np.array_equal(r("obj_geo")[k], np.array([list(o.bmin), list(o.bmax), list(o.cs), list(o.rcp)], np.float32))
        assert r("obj_first")[k] == o.cell_off
    assert tuple(r("top_res")) == tuple(ob.top.res)
    assert np.array_equal(r("top_geo"), np.array([list(ob.top.bmin), list(ob.top.bmax), list(ob.top.cs),
                                                  list(ob.top.rcp)], np.float32))
    rc, rl = cell_lists(r("top_cells"), r("inst_ids"))
    oc, ol = cell_lists(ob.top_cells, ob.inst_ids)
    assert np.array_equal(rc, oc) and np.array_equal(rl, ol)
    # object cells: identical but for boundary-layer moves of a few triangles
    rcl, rp = r("obj_cells"), r("prims")
    ocl, op = ob.obj_cells, ob.prims
    assert rcl.shape == ocl.shape
    ref_cells, orc_cells = {}, {}
    for c in range(rcl.shape[0]):
        for t in rp[rcl[c, 0]:rcl[c, 1]]:
            ref_cells.setdefault(int(t), set()).add(c)
        for t in op[ocl[c, 0]:ocl[c, 1]]:
            orc_cells.setdefault(int(t), set()).add(c)
    assert set(ref_cells) == set(orc_cells) == set(range(z["faces"].shape[0]))
    moved = [t for t in ref_cells if ref_cells[t] != orc_cells[t]]
    assert len(moved) <= 0.05 * len(ref_cells)   # heightfield tiles put many vertices on cell planes
    firsts = [ob.objs[k].cell_off for k in range(len(z["counts"]))]
    for t in moved:
        k = int(np.searchsorted(firsts, min(orc_cells[t]), side="right") - 1)
        o = ob.objs[k]
        rx, ry = o.res[0], o.res[1]

        def xyz(c):
            c -= o.cell_off
            return np.array([c % rx, (c // rx) % ry, c // (rx * ry)])
        a = np.array([xyz(c) for c in ref_cells[t]])
        b = np.array([xyz(c) for c in orc_cells[t]])
        assert np.all(np.abs(a.min(0) - b.min(0)) <= 1) and np.all(np.abs(a.max(0) - b.max(0)) <= 1)
    # hits: the same instance and triangle for every ray; t within the precision the
    # reference's reciprocal-derived directions allow
    hi, ht, t, _, _ = oracle.hier_trace(ob, z["ray_org"], z["ray_dir"])
    ri = r("hit_inst").astype(np.int64)
    ri[ri == 0xFFFFFFFF] = -1
    rt = r("hit_tri").astype(np.int64)
    rt[rt == 0xFFFFFFFF] = -1
    assert np.array_equal(ri, hi) and np.array_equal(rt, ht)
    hit = hi >= 0
    assert hit.sum() > 1000
    rel = np.abs(r("hit_t")[hit] - t[hit]) / np.abs(t[hit])
    assert rel.max() <= (5e-6 if variant == "strict" else 2e-4)
