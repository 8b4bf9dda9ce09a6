"""Scene input, ray files and image output (host code of the library, no GPU):
the reference's scene.cfg / OBJ / camera / light formats, .rays files, PNG and PFM."""
import struct
import zlib

import numpy as np
import pytest

from happyray_b200 import HRError
from happyray_b200 import scenes as S
from happyray_b200 import sceneio as IO


def write_obj(path, v, f, extra=""):
    with open(path, "w") as fh:
        fh.write("# test mesh\n" + extra)
        for p in v:
            fh.write("v %.9g %.9g %.9g\n" % tuple(p))
        for t in f:
            fh.write("f %d %d %d\n" % tuple(int(i) + 1 for i in t))


def test_obj_statement_forms(hrlib, tmp_path):
    (tmp_path / "scene.mtl").write_text("newmtl red\nKd 0.8 0.2 0.5\n")
    p = tmp_path / "forms.obj"
    p.write_text(
        "# comment line\n"
        "mtllib scene.mtl\n"
        "o thing\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0   # trailing comment\n"
        "vn 0 0 1\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n"
        "g group\ns 1\nusemtl red\n"
        "f 1 2 3\n"
        "f 1/1 2/2 3/3 4/4\n"          # quad: fanned from its first corner
        "f 1//1 3//1 4//1\n"
        "f 1/1/1 2/2/1 4/4/1\n"
        "v 2 0 0\nv 2 1 0\nv 3 1 0\n"
        "f -3 -2 -1\n"                 # relative indices
        "l 5 6\n"                      # a line: no triangle
        "l 5 6 7\n"                    # three corners make a triangle (as the reference)
        "fo 1 2 4\n")
    sc = IO.load_obj(str(p))
    assert sc.keyframes.shape == (1, 7, 3)
    assert np.array_equal(sc.keyframes[0, 4], [2, 0, 0])
    want = [[0, 1, 2], [0, 1, 2], [0, 2, 3], [0, 2, 3], [0, 1, 3], [4, 5, 6], [4, 5, 6], [0, 1, 3]]
    assert np.array_equal(sc.faces, np.array(want, np.uint32))
    # the file's one normal, then a geometric normal for each face without normal indices
    # (WFObjectReader.cpp:602-614), in face order
    assert sc.normals.shape == (7, 3)
    assert np.array_equal(sc.normal_idx, [[1, 1, 1], [2, 2, 2], [3, 3, 3], [0, 0, 0], [0, 0, 0], [4, 4, 4], [5, 5, 5],
                                          [6, 6, 6]])
    assert np.allclose(sc.normals, [[0, 0, 1]] * 4 + [[0, 0, -1]] * 2 + [[0, 0, 1]])   # 5 6 7 winds clockwise
    # "usemtl red" precedes every face: Default, then red with mean(min(Kd, 0.99))
    assert np.allclose(sc.albedo, [0.6774, 0.5]) and np.array_equal(sc.materials, [1] * 8)


def expected_geometric_normal(v, t):
    n = np.cross(v[t[1]] - v[t[0]], v[t[2]] - v[t[0]])
    return n / np.linalg.norm(n)


def test_obj_normals_and_materials(hrlib, tmp_path):
    """vn with global, relative and partial normal indices; usemtl switches; a .mtl whose
    unknown newmtl keeps the earlier selection (readMtlLib, WFObjectReader.cpp:160-170) and
    whose short Kd line is ignored; a file without vn keeps no normals."""
    (tmp_path / "m.mtl").write_text(
        "# materials\nnewmtl blue\nKd 0.1 0.2 0.3\nKs 1 1 1\nnewmtl unused\nKd 2 2 2\n"
        "newmtl green\nkd 0.25 1.0 0.5\nnewmtl grey\nKd 0.5 0.5\n")
    (tmp_path / "n.obj").write_text(
        "mtllib m.mtl\n"
        "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\n"
        "vn 1 0 0\nvn 0 1 0\nvn 0 0 1\n"
        "f 1//1 2//2 3//3\n"          # Default
        "usemtl blue\n"
        "f 1/1/-3 2/1/-2 4/1/-1\n"    # relative normal indices
        "usemtl green\n"
        "f 1//3 3 4//1\n"             # one corner without a normal index
        "usemtl blue\n"
        "f 2 3 4\n"
        "usemtl grey\n"
        "f 1 3 2\n")
    sc = IO.load_obj(str(tmp_path / "n.obj"))
    v = sc.keyframes[0]
    assert sc.normals.shape == (6, 3)
    assert np.array_equal(sc.normal_idx, [[0, 1, 2], [0, 1, 2], [2, 3, 0], [4, 4, 4], [5, 5, 5]])
    for k, t in zip((3, 4, 5), sc.faces[2:]):
        assert np.allclose(sc.normals[k], expected_geometric_normal(v.astype(np.float64), t), atol=1e-6)
    # Default, blue, green, grey ("unused" is not a material of the OBJ: its Kd 2 2 2 lands
    # on blue, the selection it left in place; grey's two-number Kd is ignored)
    assert np.allclose(sc.albedo, [0.6774, 0.99, (0.25 + 0.99 + 0.5) / 3, 0.0])
    assert np.array_equal(sc.materials, [0, 1, 2, 1, 3])
    (tmp_path / "plain.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    sc = IO.load_obj(str(tmp_path / "plain.obj"))
    assert sc.normals is None and sc.albedo is None
    (tmp_path / "nomtl.obj").write_text("mtllib missing.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(HRError) as ei:
        IO.load_obj(str(tmp_path / "nomtl.obj"))
    assert "missing.mtl" in str(ei.value)
    (tmp_path / "badn.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//2 3//1\n")
    with pytest.raises(HRError) as ei:
        IO.load_obj(str(tmp_path / "badn.obj"))
    assert "normal index" in str(ei.value)


def test_obj_normals_materials_parallel_parse(hrlib, tmp_path):
    """Normals, relative normal indices and material switches spread over many line chunks
    parse the same with 1 and 8 threads, and as a plain serial reading of the file says."""
    rng = np.random.default_rng(5)
    nv, nt = 60_000, 120_000
    v = rng.random((nv, 3), dtype=np.float32)
    nrm = rng.normal(size=(nv, 3)).astype(np.float32)
    f = rng.integers(0, nv, (nt, 3))
    (tmp_path / "mats.mtl").write_text("".join("newmtl m%d\nKd %.3f %.3f %.3f\n" % (i, i / 10, i / 20, 0.3)
                                               for i in range(8)))
    lines = ["mtllib mats.mtl\n"]
    lines += ["v %.9g %.9g %.9g\nvn %.9g %.9g %.9g\n" % (tuple(p) + tuple(q)) for p, q in zip(v, nrm)]
    want_mat = np.zeros(nt, np.uint32)
    want_nid = np.zeros((nt, 3), np.int64)
    order, cur = [], 0
    for i, t in enumerate(f):
        if i % 997 == 0:
            m = int(rng.integers(0, 8))
            lines.append("usemtl m%d\n" % m)
            if m not in order:
                order.append(m)
            cur = order.index(m) + 1
        want_mat[i] = cur
        if i % 2:
            lines.append("f %d//%d %d//%d %d//%d\n" % (t[0] + 1, t[0] + 1, t[1] + 1, t[1] + 1, t[2] + 1, t[2] + 1))
        else:                          # relative to the nv normals read so far
            lines.append("f %d//%d %d//%d %d//%d\n" % (t[0] + 1, t[0] - nv, t[1] + 1, t[1] - nv, t[2] + 1, t[2] - nv))
        want_nid[i] = t
    p = tmp_path / "big.obj"
    p.write_text("".join(lines))
    assert p.stat().st_size > 8 << 20
    a = IO.load_obj(str(p), threads=1)
    b = IO.load_obj(str(p), threads=8)
    for x, y in ((a.normals, b.normals), (a.normal_idx, b.normal_idx), (a.albedo, b.albedo),
                 (a.materials, b.materials)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.normals, nrm) and np.array_equal(a.normal_idx, want_nid)
    assert np.array_equal(a.materials, want_mat)
    kd = np.minimum(np.array([[i / 10, i / 20, 0.3] for i in range(8)], np.float32), 0.99).mean(axis=1)
    assert np.allclose(a.albedo, np.concatenate([[0.6774], kd[order]]), atol=1e-6)


def test_obj_parallel_parse_matches_serial(hrlib, tmp_path):
    v, f = S.heightfield(257, 3)           # 131,072 triangles, a multi-chunk file
    p = tmp_path / "big.obj"
    write_obj(p, v, f)
    assert p.stat().st_size > 4 << 20
    a = IO.load_obj(str(p), threads=1)
    b = IO.load_obj(str(p), threads=8)
    assert np.array_equal(a.keyframes, b.keyframes) and np.array_equal(a.faces, b.faces)
    assert np.array_equal(a.keyframes[0], v) and np.array_equal(a.faces, f)


@pytest.mark.parametrize("text,msg", [("v 1 2\n", "line 2"), ("v 0 0 0\nf 1 2 9\n", "out of range"),
                                      ("v 0 0 0\nf 1 x 2\n", "bad face index")])
def test_obj_errors(hrlib, tmp_path, text, msg):
    p = tmp_path / "bad.obj"
    p.write_text("# bad\n" + text)
    with pytest.raises(HRError) as ei:
        IO.load_obj(str(p))
    assert ei.value.status == 1 and msg in str(ei.value)
    with pytest.raises(HRError):
        IO.load_obj(str(tmp_path / "missing.obj"))


def test_scene_cfg_key_frames_camera_lights(hrlib, tmp_path):
    v, f = S.heightfield(9, 0)
    frames = S.curl_keyframes(v, 12, amp=0.02, octaves=2, seed=1)
    (tmp_path / "anim").mkdir()
    for k in range(12):                    # 12 frames: names padded to 2 digits
        write_obj(tmp_path / "anim" / ("hf_%02d.obj" % k), frames[k], f)
    (tmp_path / "camera.cfg").write_text(
        "# camera\nposition 0.5 -0.8 0.9\norientation 0 1 -0.5\nup 0 0 1\nrotation 0 0 90\nresX 320\nresY 200\nFOV 45\n")
    (tmp_path / "light.cfg").write_text(
        "position 0.4 0.4 1\nintensity 10 20 30\nedge1 0.2 0 0\nedge2 0 0.2 0\n"
        "position 0 0 2\nnormal 0 0 -1\nintensity 1 1 1\nedge1 1 0 0\nedge2 0 1 0\n")
    (tmp_path / "scene.cfg").write_text(
        "# animated\nframe prefix = anim/hf_\nframe suffix = .obj\nnumber of frames = 12\nframe step = 0.4\n"
        "camera = camera.cfg\nlight = light.cfg\nunknown key = 1\n")
    sc = IO.load_scene(str(tmp_path / "scene.cfg"))
    assert sc.keyframes.shape == (12, v.shape[0], 3)
    assert np.array_equal(sc.keyframes, frames) and np.array_equal(sc.faces, f)
    assert sc.frame_step == pytest.approx(0.4)
    c = sc.camera
    assert (c["res_x"], c["res_y"], c["fov"]) == (320, 200, 45.0)
    # 90 degrees about z with CameraManager::rotate's column formulas: (x, y, z) -> (y, -x, z)
    assert np.allclose(c["orientation"], [1, 0, -0.5], atol=1e-6) and np.allclose(c["up"], [0, 0, 1], atol=1e-6)
    assert len(sc.lights) == 2
    assert np.allclose(sc.lights[0].normal, [0, 0, 1]) and np.allclose(sc.lights[0].intensity, [10, 20, 30])
    assert np.allclose(sc.lights[1].normal, [0, 0, -1])


def test_scene_cfg_static_objs(hrlib, tmp_path):
    v1, f1 = S.heightfield(5, 0)
    v2, f2 = S.icosphere(1)
    write_obj(tmp_path / "a.obj", v1, f1)
    write_obj(tmp_path / "b.obj", np.asarray(v2, np.float32), f2)
    (tmp_path / "scene.cfg").write_text("obj = a.obj\nscene = b.obj\n")
    sc = IO.load_scene(str(tmp_path / "scene.cfg"))
    assert sc.keyframes.shape[0] == 1 and sc.camera is None and not sc.lights
    assert np.array_equal(sc.faces, np.concatenate([f1, f2 + v1.shape[0]]))


def test_scene_cfg_normals_materials(hrlib, tmp_path):
    """A static scene of two OBJs, the first without vn or materials, the second with both:
    the first file's faces get geometric normals and "Default"; the second's normal indices
    move past them.  Key frames keep the first frame's normals and the last's materials."""
    (tmp_path / "a.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nf 1 3 2\n")
    (tmp_path / "b.mtl").write_text("newmtl red\nKd 0.9 0.3 0.3\n")
    (tmp_path / "b.obj").write_text("mtllib b.mtl\nv 0 0 1\nv 1 0 1\nv 0 1 1\nvn 0 1 0\nvn 1 0 0\n"
                                    "usemtl red\nf 1//2 2//1 3//2\n")
    (tmp_path / "scene.cfg").write_text("obj = a.obj\nobj = b.obj\n")
    sc = IO.load_scene(str(tmp_path / "scene.cfg"))
    assert np.array_equal(sc.faces, [[0, 1, 2], [0, 2, 1], [3, 4, 5]])
    assert np.array_equal(sc.normals, [[0, 1, 0], [1, 0, 0], [0, 0, 1], [0, 0, -1]])
    assert np.array_equal(sc.normal_idx, [[2, 2, 2], [3, 3, 3], [1, 0, 1]])
    assert np.allclose(sc.albedo, [0.6774, 0.5]) and np.array_equal(sc.materials, [0, 0, 1])
    (tmp_path / "anim").mkdir()
    for k, (nz, mat) in enumerate(((1, "red"), (-1, "blue"))):
        (tmp_path / "anim" / ("f%d.obj" % k)).write_text(
            "mtllib ../b.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 %d\nusemtl %s\nf 1//1 2//1 3//1\n" % (nz, mat))
    (tmp_path / "anim.cfg").write_text("frame prefix = anim/f\nframe suffix = .obj\nnumber of frames = 2\n")
    sc = IO.load_scene(str(tmp_path / "anim.cfg"))
    assert np.array_equal(sc.normals, [[0, 0, 1]]) and np.array_equal(sc.normal_idx, [[0, 0, 0]])
    assert sc.albedo.tolist() == pytest.approx([0.6774, 0.0]) and np.array_equal(sc.materials, [1])


def test_ray_and_hit_files(hrlib, tmp_path):
    rng = np.random.default_rng(0)
    o = rng.normal(size=(1000, 3)).astype(np.float32)
    d = rng.normal(size=(1000, 3)).astype(np.float32)
    p = tmp_path / "q.rays"
    IO.write_rays(str(p), o, d)
    raw = np.fromfile(p, np.float32).reshape(-1, 6)           # the reference's layout
    assert np.array_equal(raw[:, :3], o) and np.array_equal(raw[:, 3:], d)
    o2, d2 = IO.read_rays(str(p))
    assert np.array_equal(o2, o) and np.array_equal(d2, d)
    (tmp_path / "bad.rays").write_bytes(b"\0" * 25)
    with pytest.raises(HRError):
        IO.read_rays(str(tmp_path / "bad.rays"))
    hid = rng.integers(-1, 100, 1000).astype(np.int32)
    t, u, v = [rng.random(1000).astype(np.float32) for _ in range(3)]
    IO.write_hits(str(tmp_path / "q.hits"), hid, t, u, v)
    rec = np.fromfile(tmp_path / "q.hits", dtype=[("id", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
    assert np.array_equal(rec["id"], hid) and np.array_equal(rec["t"], t) and np.array_equal(rec["v"], v)


def read_png(path):
    b = path.read_bytes()
    assert b[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(b):
        n, typ = struct.unpack(">I4s", b[pos:pos + 8])
        data = b[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", b[pos + 8 + n:pos + 12 + n])[0]
        assert crc == zlib.crc32(typ + data) & 0xFFFFFFFF
        chunks.setdefault(typ, b"")
        chunks[typ] += data
        pos += 12 + n
    w, h, depth, ctype = struct.unpack(">IIBB", chunks[b"IHDR"][:10])
    raw = zlib.decompress(chunks[b"IDAT"])                     # checks the Adler-32 too
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 3 * w)
    assert (depth, ctype) == (8, 2) and np.all(rows[:, 0] == 0)
    return rows[:, 1:].reshape(h, w, 3)


def test_png_and_pfm(hrlib, tmp_path):
    rng = np.random.default_rng(1)
    img = rng.uniform(-0.5, 1.5, (37, 150, 3)).astype(np.float32)   # values outside [0, 1] are clamped
    img[0, 0, 0] = np.nan
    IO.write_image(str(tmp_path / "a.png"), img, 150, 37)
    got = read_png(tmp_path / "a.png")
    want = (np.clip(np.nan_to_num(img, nan=0.0), 0, 1) * np.float32(255)).astype(np.uint8)
    assert np.array_equal(got, want)
    big = rng.random((300, 400, 3)).astype(np.float32)             # > 65,535 raw bytes: several stored blocks
    IO.write_image(str(tmp_path / "b.png"), big, 400, 300)
    assert np.array_equal(read_png(tmp_path / "b.png"), (big * np.float32(255)).astype(np.uint8))
    IO.write_image(str(tmp_path / "c.pfm"), img, 150, 37, IO.IMAGE_PFM)
    b = (tmp_path / "c.pfm").read_bytes()
    head = b"PF\n150 37\n-1.0\n"
    assert b[:len(head)] == head
    data = np.frombuffer(b[len(head):], "<f4").reshape(37, 150, 3)[::-1]
    assert np.array_equal(data, img, equal_nan=True)
    with pytest.raises(HRError):
        IO.write_image(str(tmp_path / "d.png"), img, 150, 36)
