"""Golden vectors of the reference's OWN grid build and traversal.

The reference (javorkk/happyray) has no CPU code path, no tests and no fixtures for the
build and traversal, so its kernels are run themselves: oracle/ref_pin/ref_pin.cu is a
harness that includes the reference's build kernels and traversers from its source tree
(compiled in place by `make -C oracle/ref_pin` into oracle/_ref/; nothing is copied) and
drives them in the order its builders launch them.  This script writes small seeded
inputs, runs both harness builds on a GPU and stores what the reference computed:

    python tests/golden/make_ref_golden.py OUT_DIR

  ref_<case>.npz   inputs (vertices, triangles, rays, densities) and, per harness build
                   (strict = IEEE arithmetic without FMA contraction, the oracle's contract;
                   fast = the reference's own -use_fast_math build), the grid parameters,
                   cells, leaves, primitive lists and hits.

  ref_hier_<case>.npz   the instanced two-level grid hierarchy: objects, instances and
                   rays in; per harness build (oracle/ref_pin/ref_pin_hier.cu, the
                   reference's TLGridHierarchySortBuilder and TLGridHierarchyTraverser)
                   the object grids, object cells, triangle lists, instance grid, instance
                   lists and hits (`--hier` writes only these).

tests/test_oracle.py::test_oracle_matches_reference_golden and
tests/test_hier_oracle.py::test_oracle_hier_matches_reference_golden compare the oracle
with these files on the CPU.  Test infrastructure only.
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from happyray_b200 import scenes as S  # noqa: E402
import oracle as O  # noqa: E402

BIN = {"strict": ROOT / "oracle" / "_ref" / "ref_pin_strict", "fast": ROOT / "oracle" / "_ref" / "ref_pin_fast"}
HIER_BIN = {"strict": ROOT / "oracle" / "_ref" / "ref_pin_hier_strict",
            "fast": ROOT / "oracle" / "_ref" / "ref_pin_hier_fast"}


def cases():
    """(name, kind, exact, density, leaf density, vertices, triangles, camera)"""
    hv, hf = S.heightfield(33, 0)                       # 2,048 triangles
    cv, cf = S.clusters(12_000, seed=7)
    return [
        ("ug_exact_heightfield", 0, 1, 5.0, 0.0, hv, hf, S.camera_c1((64, 64))),
        ("ug_bbox_heightfield", 0, 0, 5.0, 0.0, hv, hf, S.camera_c1((64, 64))),
        ("ug_exact_clusters", 0, 1, 5.0, 0.0, cv, cf, S.camera_at_bounds(cv, (64, 48))),
        ("tl_clusters", 1, 0, 0.0625, 2.0, cv, cf, S.camera_at_bounds(cv, (64, 48))),
        ("tl_clusters_dense", 1, 0, 0.25, 4.0, cv, cf, S.camera_at_bounds(cv, (64, 48))),
        ("tl_heightfield", 1, 0, 0.0625, 2.0, hv, hf, S.camera_c1((64, 64))),
    ]


def write_input(path, kind, exact, dens, leaf, v, f, org, d):
    v = np.ascontiguousarray(v, np.float32)
    f = np.ascontiguousarray(f, np.uint32)
    rays = np.ascontiguousarray(np.concatenate([org, d], axis=1), np.float32)
    with open(path, "wb") as fh:
        fh.write(b"HRP1")
        fh.write(np.array([kind, exact, v.shape[0], f.shape[0], rays.shape[0]], np.uint32).tobytes())
        fh.write(np.array([dens, leaf], np.float32).tobytes())
        fh.write(v.tobytes())
        fh.write(f.tobytes())
        fh.write(rays.tobytes())


def read_output(path, nrays):
    b = Path(path).read_bytes()
    o = 0

    def take(dtype, n):
        nonlocal o
        a = np.frombuffer(b, dtype, n, o)
        o += a.nbytes
        return a.copy()

    res = take(np.int32, 3)
    geo = take(np.float32, 12).reshape(4, 3)
    nc = int(take(np.uint32, 1)[0])
    cells = take(np.uint32, 2 * nc).reshape(-1, 2)
    nl = int(take(np.uint32, 1)[0])
    leaves = take(np.uint32, 2 * nl).reshape(-1, 2)
    npr = int(take(np.uint32, 1)[0])
    prims = take(np.uint32, npr)
    hits = np.frombuffer(b, np.uint32, 2 * nrays, o).reshape(-1, 2)
    return {"res": res, "bmin": geo[0], "bmax": geo[1], "cs": geo[2], "rcp": geo[3], "cells": cells,
            "leaves": leaves, "prims": prims, "hit_id": hits[:, 0].copy(), "hit_t": hits[:, 1].copy().view(np.float32)}


def hier_cases():
    """(name, top density, object density, seed, objects, instances, triangle range, scales)"""
    return [
        ("hier_small", 1.2, 1.2, 3, 4, 48, (80, 1500), (0.08, 0.25)),
        ("hier_dense", 0.5, 3.0, 5, 8, 300, (80, 4000), (0.03, 0.12)),
    ]


def hier_rays(inst, n, seed):
    rng = np.random.default_rng(seed)
    c = 0.5 * (inst["bmin"] + inst["bmax"])
    tgt = c[rng.integers(0, len(inst), n)] + rng.normal(0, 0.03, (n, 3))
    org = rng.uniform(-0.5, 1.5, (n, 3)).astype(np.float32)
    return org, (tgt - org).astype(np.float32)


def write_hier_input(path, top, leaf, v, f, counts, inst, org, d):
    rays = np.ascontiguousarray(np.concatenate([org, d], axis=1), np.float32)
    with open(path, "wb") as fh:
        fh.write(b"HRH1")
        fh.write(np.array([v.shape[0], f.shape[0], len(counts), len(inst), rays.shape[0]], np.uint32).tobytes())
        fh.write(np.array([top, leaf], np.float32).tobytes())
        fh.write(np.ascontiguousarray(v, np.float32).tobytes())
        fh.write(np.ascontiguousarray(f, np.uint32).tobytes())
        fh.write(np.ascontiguousarray(counts, np.uint32).tobytes())
        fh.write(np.ascontiguousarray(inst, S.INSTANCE_DTYPE).tobytes())
        fh.write(rays.tobytes())


def read_hier_output(path, nobj, nrays):
    b = Path(path).read_bytes()
    o = 0

    def take(dtype, n):
        nonlocal o
        a = np.frombuffer(b, dtype, n, o)
        o += a.nbytes
        return a.copy()

    res, geo, first = [], [], []
    for _ in range(nobj):
        res.append(take(np.int32, 3))
        geo.append(take(np.float32, 12))
        first.append(take(np.uint32, 1)[0])
    out = {"obj_res": np.array(res), "obj_geo": np.array(geo).reshape(-1, 4, 3), "obj_first": np.array(first)}
    out["obj_cells"] = take(np.uint32, 2 * int(take(np.uint32, 1)[0])).reshape(-1, 2)
    out["prims"] = take(np.uint32, int(take(np.uint32, 1)[0]))
    out["top_res"] = take(np.int32, 3)
    out["top_geo"] = take(np.float32, 12).reshape(4, 3)
    out["top_cells"] = take(np.uint32, 2 * int(take(np.uint32, 1)[0])).reshape(-1, 2)
    out["inst_ids"] = take(np.uint32, int(take(np.uint32, 1)[0]))
    hits = np.frombuffer(b, np.uint32, 3 * nrays, o).reshape(-1, 3)
    out["hit_inst"], out["hit_tri"] = hits[:, 0].copy(), hits[:, 1].copy()
    out["hit_t"] = hits[:, 2].copy().view(np.float32)
    return out


def main_hier(out_dir: Path):
    out_dir.mkdir(parents=True, exist_ok=True)
    for name, top, leaf, seed, nobj, ninst, tri_range, scales in hier_cases():
        v, f, counts, inst = S.instanced_scene(nobj, ninst, seed=seed, tri_range=tri_range, scale_range=scales)
        org, d = hier_rays(inst, 4000, seed + 11)
        rec = {"vertices": v, "faces": f, "counts": counts, "instances": inst, "ray_org": org, "ray_dir": d,
               "top_density": np.float32(top), "object_density": np.float32(leaf)}
        with tempfile.TemporaryDirectory() as td:
            inp = Path(td) / "in.bin"
            write_hier_input(inp, top, leaf, v, f, counts, inst, org, d)
            for var, exe in HIER_BIN.items():
                outp = Path(td) / f"out_{var}.bin"
                r = subprocess.run([str(exe), str(inp), str(outp)], capture_output=True, text=True, timeout=120)
                if r.returncode != 0:
                    raise SystemExit(f"{name} {var}: {r.stderr.strip()}")
                print(name, var, r.stdout.strip(), flush=True)
                for k, a in read_hier_output(outp, len(counts), org.shape[0]).items():
                    rec[f"{var}_{k}"] = a
        np.savez_compressed(out_dir / f"ref_{name}.npz", **rec)


def main(out_dir: Path):
    out_dir.mkdir(parents=True, exist_ok=True)
    O.build()
    for name, kind, exact, dens, leaf, v, f, cam in cases():
        oc = O.camera(cam["position"], cam["orientation"], cam["up"], cam["fov"], cam["res_x"], cam["res_y"])
        org, d = O.primary_rays(oc)
        rec = {"vertices": np.asarray(v, np.float32), "faces": np.asarray(f, np.uint32), "ray_org": org,
               "ray_dir": d, "kind": np.int32(kind), "exact": np.int32(exact), "density": np.float32(dens),
               "leaf_density": np.float32(leaf)}
        with tempfile.TemporaryDirectory() as td:
            inp = Path(td) / "in.bin"
            write_input(inp, kind, exact, dens, leaf, v, f, org, d)
            for var, exe in BIN.items():
                outp = Path(td) / f"out_{var}.bin"
                r = subprocess.run([str(exe), str(inp), str(outp)], capture_output=True, text=True, timeout=120)
                if r.returncode != 0:
                    raise SystemExit(f"{name} {var}: {r.stderr.strip()}")
                print(name, var, r.stdout.strip(), flush=True)
                for k, a in read_output(outp, org.shape[0]).items():
                    rec[f"{var}_{k}"] = a
        np.savez_compressed(out_dir / f"ref_{name}.npz", **rec)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a != "--hier"]
    out = Path(args[0]) if args else Path(__file__).resolve().parent
    if "--hier" in sys.argv[1:]:
        main_hier(out)
    else:
        main(out)
        main_hier(out)
