#!/usr/bin/env python
"""Benchmark of the happyray hot path on B200: per-frame grid rebuild + traversal.

Default workload (the configuration the headline metric is quoted on):
  c2: two-level grid over 1,048,576 seeded triangles (64 clusters of level-4 icospheres +
      ground plane), top density 1/16, leaf density 2; 1920x1080 primary rays + 8 cosine AO
      rays per hit, AO radius 0.1 x bounds diagonal, PCG32 per pixel.
A step is one frame: device key-frame interpolation + bounds, two-level grid rebuild,
primary + AO traversal.  value = rays traced / step time (Mrays/s), whole job over all GPUs.
Other workloads: c1 (uniform grid, 129x129 heightfield, 256x256 primary rays), c3
(2,097,152 triangles, 16 curl-noise key frames, rebuild per frame, 1280x720 path tracing),
c4 (256 scenes of 1k-500k triangles batched: one segmented build + one persistent
render launch in a CUDA graph, against the per-scene path on the same scenes) and c5
(64 resident animated scenes served under Poisson arrivals, continuous batching against
the serial per-scene path; p50/p99 latency).

c2 and c3 lines also carry `fast_arith`: the same steps through libhappyray_b200_fast.so
(traversal kernels with FMA contraction and approximate division, IEEE grid build), its
Mrays/s and its image on the CPU baseline's frame against the oracle's.

Multi-GPU (torchrun): independent replicas, one per GPU (the path has no exchange step).
`--impl reference` times the CPU restatement of the reference's build + traversal
(oracle/, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import signal
import statistics
import subprocess
import tempfile
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s (AO, PT) and grid rebuild ms per frame; p50/p99 request latency"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` on `workload` from its committed ncu summary
    (profiles/<kernel>__<workload>.md, line 'dram_bytes_per_launch: N'), or None."""
    prof = ROOT / "profiles" / f"{kernel}__{workload}.md"
    if prof.exists():
        for line in prof.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    return None


def l2_read_gbs(stream=None):
    """L2-resident read rate measured on this device by the library's probe
    (hr_probe_l2_read: one kernel reads a 32 MiB buffer 50 times through L2).  The
    traversal kernels' working sets live mostly in L2, so their algorithmic bytes are also
    reported against this rate."""
    import ctypes as C
    from happyray_b200 import _lib
    out = C.c_double(0.0)
    st = _lib.load().hr_probe_l2_read(C.c_void_p(stream.cuda_stream if stream is not None else 0), C.byref(out))
    return out.value if st == 0 else None


def workload(name: str):
    from happyray_b200 import scenes as S
    if name == "c1":
        v, f = S.heightfield(129, 0)
        return dict(name="c1_uniform_primary_heightfield_256", v=v, f=f, kind=0, exact=True, ug=5.0,
                    cam=S.camera_c1((256, 256)), mode=0, frames=None)
    if name == "c2":
        v, f = S.clusters(1_048_576, seed=0)
        return dict(name="c2_two_level_ao_1M_1080p", v=v, f=f, kind=1, top=0.0625, leaf=2.0,
                    cam=S.camera_at_bounds(v, (1920, 1080)), mode=3, ao=8, frames=None)
    if name == "c3":
        v, f = S.clusters(2_097_152, seed=0)
        frames = S.curl_keyframes(v, 16, amp=0.02, octaves=4, seed=0)
        return dict(name="c3_two_level_keyframe_pt_2M_720p", v=v, f=f, kind=1, top=0.0625, leaf=2.0,
                    cam=S.camera_at_bounds(v, (1280, 720)), mode=1, bounces=4, frames=frames)
    raise SystemExit(f"unknown config {name}")


def algorithmic_build_bytes(gi, nv, ntri, lerp=True):
    """Bytes read + written once by each stage (per-unit figures of the build roofline):
    uniform 40V + 2M + 36P + 8C, two-level 104V + 48N + 52 P_top + 44 C_top + 36 P_leaf + 8 C_leaf,
    M = 12N + 16V; the 40V interpolation term is kept since every step interpolates."""
    if gi["kind"] == 0:
        M = 12 * ntri + 16 * nv
        return (40 * nv if lerp else 0) + 2 * M + 36 * gi["num_pairs"] + 8 * gi["num_cells"]
    return (104 * nv + 48 * ntri + 52 * gi["num_top_pairs"] + 44 * gi["num_cells"] + 36 * gi["num_pairs"]
            + 8 * gi["num_leaves"] - (0 if lerp else 40 * nv))


def trace_bytes(rays, cells, tests):
    """Algorithmic traversal bytes: per ray 28 B ray + 16 B hit, 8 B per cell or leaf visited,
    52 B per triangle test (4 B reference + 12 B indices + 36 B vertices)."""
    return 44 * rays + 8 * cells + 52 * tests


class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        out = Path(tempfile.gettempdir())
        self.path = out / f"clocks_gpu{self.index}.csv"
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.path or not self.path.exists():
            return None
        rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    import torch
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, ws, local


def max_over_ranks(x: float, ws: int) -> float:
    """Largest value over the ranks -- the slowest replica's device time -- or x itself at
    N = 1.  Works on a NCCL (GPU tensor) or gloo (CPU tensor) process group."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank_step: float, steps: int, total_ms: float, ws: int) -> float:
    """Whole-job throughput in millions of units per second: the units every replica
    processed over the slowest replica's time (weak scaling: fixed work per GPU)."""
    return ws * units_per_rank_step * steps / (total_ms * 1e-3) / 1e6


def baseline_frame(W):
    """The frame the CPU baseline builds and renders: key frames 0 and 1 blended half-way
    for an animated workload, the static mesh otherwise (first frame, second frame, weight)."""
    frames = W["frames"]
    if frames is not None:
        return frames[0], frames[1], 0.5
    return W["v"], W["v"], 1.0


def cpu_baseline(W, kind_budget_s=25.0, keep=None):
    """The oracle (CPU restatement of the reference's build and traversal) on a bounded
    sample of the workload, all host threads: full build + a strided pixel sample, scaled.
    With keep (a dict), the oracle's grid and outputs are stored there for the parity check."""
    import oracle as O
    f = W["f"]
    f1, f2, coeff = baseline_frame(W)
    t0 = time.perf_counter()
    v4, bmin, bmax = O.lerp_bounds(f1, f2, coeff)
    if W["kind"] == 0:
        b = O.build_ug(v4, f, bmin, bmax, W["ug"], W["exact"])
    else:
        b = O.build_tl(v4, f, bmin, bmax, W["top"], W["leaf"])
    t_build = time.perf_counter() - t0
    cam = W["cam"]
    oc = O.camera(cam["position"], cam["orientation"], cam["up"], cam["fov"], cam["res_x"], cam["res_y"])
    npx = cam["res_x"] * cam["res_y"]
    stride = 1 if W["mode"] != 1 else 2
    t1 = time.perf_counter()
    if W["mode"] == 3:
        out, rays = O.render_ao(b, oc, W["ao"], float(np.float32(0.1) * b.diag()), 0x853c49e6748fea9b,
                                pixel_stride=stride)
    elif W["mode"] == 1:
        out, rays = O.render_pt(b, oc, O.make_light(), W["bounces"], 0.7, float(np.float32(1e-4) * b.diag()),
                                0x853c49e6748fea9b, pixel_stride=stride)
    else:
        org, d = O.primary_rays(oc)
        out = O.trace(b, org[::stride], d[::stride])
        rays = org[::stride].shape[0]
    t_trace = time.perf_counter() - t1
    if keep is not None:
        keep.update(grid=b, out=out, stride=stride)
    sampled = len(range(0, npx, stride))
    scale = npx / sampled
    est = t_build + t_trace * scale
    return {"value": rays * scale / est / 1e6, "unit": "Mrays/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"full build ({t_build * 1e3:.0f} ms) + every {stride}th pixel ({sampled} px, "
                      f"{rays} rays, {t_trace * 1e3:.0f} ms) scaled to the full frame",
            "build_ms": t_build * 1e3}


def gpu_parity(eng, W, keep, d_fb):
    """The CPU baseline's frame built and rendered through the library (untimed), compared
    with the oracle's grid and output: the number of differing entries of each (0 everywhere
    = bit-exact)."""
    import torch
    f1, f2, coeff = baseline_frame(W)
    eng.upload(f1, f2, W["f"], coeff)
    eng.build(W["kind"], W.get("exact", True))
    gi, cells, leaves, prims = eng.grid_download()
    b = keep["grid"]

    def ndiff(a, o):
        a, o = np.asarray(a).reshape(-1), np.asarray(o).reshape(-1)
        return int((a != o).sum()) if a.shape == o.shape else max(a.size, o.size)

    res = {"grid_cells": ndiff(cells, b.cells), "grid_prims": ndiff(prims, b.prims)}
    if b.leaves is not None:
        res["grid_leaves"] = ndiff(leaves, b.leaves)
    st = keep["stride"]
    if W["mode"] in (1, 3):
        eng.render_device(d_fb, 0, W["mode"])
        eng.sync()
        img = d_fb.view(-1, 3).cpu().numpy()
        res["pixels_compared"] = int(img[::st].shape[0])
        res["pixels_differing"] = ndiff(img[::st, 0], keep["out"][::st])
    else:
        n = W["cam"]["res_x"] * W["cam"]["res_y"]
        outs = [torch.empty(n, dtype=dt, device=d_fb.device) for dt in (torch.int32, torch.float32, torch.float32,
                                                                        torch.float32)]
        eng.trace_primary_device(*outs)
        eng.sync()
        res["rays_compared"] = int(n)
        res["hits_differing"] = sum(ndiff(o.cpu().numpy()[::st], k) for o, k in zip(outs, keep["out"]))
    res["result"] = "bit-exact" if all(v == 0 for k, v in res.items() if "differing" in k or k.startswith("grid_")) \
        else "mismatch"
    res["checked_against"] = "oracle (CPU restatement of the reference) on the CPU baseline's frame"
    return res


def rebuild_2m_prepare(dev, stream):
    """A context holding the 2,097,152-triangle key-frame mesh (16 curl-noise key frames,
    densities 1/16 : 2), with its capacities sized and its build graph captured by three
    untimed rebuilds."""
    from happyray_b200 import GRID_TWO_LEVEL, Engine
    from happyray_b200 import scenes as S
    v, f = S.clusters(2_097_152, seed=0)
    frames = S.curl_keyframes_torch(v, 16, amp=0.02, octaves=4, seed=0, device=f"cuda:{dev}")
    e = Engine(dev, stream=stream.cuda_stream)
    e.set_keyframes(frames, f)
    e.setGridDensities(0.0625, 2.0)
    for i in range(3):
        e.set_frame_time(16.0 * i / 120.0, 0.0)
        e.build(GRID_TWO_LEVEL)
    return e, v.shape[0], f.shape[0]


def rebuild_2m_keyframe(prep, stream, flush, frame_times=24):
    """Two-level rebuilds of the prepared 2M-triangle key-frame mesh at `frame_times`
    successive frame times of the 120-step cycle, each one replay of the captured build
    graph with the key-frame interpolation fused in, L2 flushed before each.  Returns the
    median rebuild time, its algorithmic bytes and the number of rebuilds timed."""
    import torch
    from happyray_b200 import GRID_TWO_LEVEL
    e, nv, ntri = prep
    ms = []
    for i in range(frame_times):
        e.set_frame_time(16.0 * ((i + 3) % 120) / 120.0, 0.0)
        with torch.cuda.stream(stream):
            flush.zero_()
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.build(GRID_TWO_LEVEL)
        z.record(stream)
        z.synchronize()
        ms.append(a.elapsed_time(z))
    gi = e.grid_info()
    return statistics.median(ms), algorithmic_build_bytes(gi, nv, ntri, lerp=True), len(ms)


def run_reference(args, W, rank, ws):
    if rank != 0:
        return
    import oracle as O
    for _ in range(args.warmup):
        cpu_baseline(W)
    vals, builds = [], []
    t0 = time.perf_counter()
    res = None
    for _ in range(args.steps):
        res = cpu_baseline(W)
        vals.append(res["value"])
        builds.append(res["build_ms"])
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall * 1e3 / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": W["name"], "triangles": int(W["f"].shape[0])}, "impl": "reference",
            "build_ms_per_frame": statistics.median(builds),
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": O.num_threads(), "kind": "port",
                             "sample": res["sample"]},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


DEFAULT_SEED = 0x853c49e6748fea9b


def batch_workload(n: int = 256, seed: int = 0):
    """Batched workload: n scenes, triangles log-uniform in [1k, 500k], heightfield or
    cluster scene (coin flip), square images log-uniform in [64^2, 512^2] pixels, primary
    rays + 4 AO rays per hit."""
    from happyray_b200 import scenes as S
    from happyray_b200.batch import SceneSpec
    raw = S.batch_scenes(n, seed)
    specs = [SceneSpec(r["v"], r["f"], r["cam"]["position"], r["cam"]["orientation"], r["cam"]["up"],
                       r["cam"]["fov"], r["cam"]["res_x"], r["cam"]["res_y"], ao_samples=4) for r in raw]
    return dict(name=f"c4_batched_{n}_scenes_primary_ao4", specs=specs)


def cpu_baseline_batch(specs, top=0.0625, leaf=2.0, budget_s=20.0):
    """The oracle on whole scenes of the batch, in order, until the time budget: full
    two-level build + AO render (4 samples) of each, all host threads."""
    import oracle as O
    rays_tot, t_tot, ns = 0, 0.0, 0
    for sp in specs:
        t0 = time.perf_counter()
        v4, bmin, bmax = O.lerp_bounds(sp.vertices, sp.vertices, 1.0)
        b = O.build_tl(v4, sp.faces, bmin, bmax, top, leaf)
        oc = O.camera(sp.position, sp.orientation, sp.up, sp.fov, sp.width, sp.height)
        _, rays = O.render_ao(b, oc, sp.ao_samples, float(np.float32(0.1) * b.diag()), DEFAULT_SEED)
        t_tot += time.perf_counter() - t0
        rays_tot += rays
        ns += 1
        if t_tot > budget_s:
            break
    return {"value": rays_tot / t_tot / 1e6, "unit": "Mrays/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"first {ns} of {len(specs)} scenes, each a full build + AO render ({rays_tot} rays, "
                      f"{t_tot:.1f} s)"}


def run_batched(args, rank, ws, local):
    """c4: the batched form (one segmented build + one persistent render launch for all
    scenes, CUDA graph) against the plain per-scene path (one hr_ctx per scene, build +
    render each) on the same scenes, densities and samples."""
    W = batch_workload()
    specs = W["specs"]
    if args.impl == "reference":
        if rank == 0:
            cb = cpu_baseline_batch(specs)
            v = cb["value"]
            print(json.dumps({"metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
                              "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                              "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                              "config": {"workload": W["name"]}, "impl": "reference", "cpu_baseline": cb,
                              "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    from happyray_b200 import GRID_TWO_LEVEL, RENDER_AO, Engine
    from happyray_b200.batch import Batch
    dev = local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    b = Batch(dev, stream=stream.cuda_stream)
    b.set_scenes(specs)
    b.set_integrator(0.1, DEFAULT_SEED)
    t0 = time.perf_counter()
    tuning = b.autotune(reps=2) if not args.no_tune else None
    tune_s = time.perf_counter() - t0
    top = tuning["top_density"] if tuning else 0.0625
    leaf = tuning["leaf_density"] if tuning else 2.0
    b.run(0)
    b.counters(reset=True)
    b.run(0)
    rays_per_step = b.counters(reset=True)[0]
    for _ in range(args.warmup):
        b.run(0)
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    l0 = b.counters()[1]
    step_ms, build_ms, render_ms = [], [], []
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()   # L2 flush between timed steps, outside the step's events
            b.run(0)
            tb, tr, tt = b.times()
            build_ms.append(tb)
            render_ms.append(tr)
            step_ms.append(tt)
        torch.cuda.synchronize()
    launches = b.counters()[1] - l0
    total_ms = max_over_ranks(sum(step_ms), ws)
    value = replica_value(rays_per_step, args.steps, total_ms, ws)

    # end to end through the public API: new vertex positions of every scene from pinned
    # host memory, build + render, every image back to pinned host memory
    e2e = None
    if not args.no_e2e:
        allv = np.concatenate([np.asarray(s.vertices, np.float32).reshape(-1, 3) for s in specs])
        hv = torch.from_numpy(allv).pin_memory().numpy()
        npx = sum(s.width * s.height for s in specs)
        himg = torch.zeros(npx * 3, dtype=torch.float32).pin_memory().numpy()
        e_ms = []
        for i in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b.set_vertices(hv)
            b.run(0)
            b.download_images(himg)
            z.record(stream)
            z.synchronize()
            if i >= args.warmup:
                e_ms.append(a.elapsed_time(z))
        et_serial = max_over_ranks(sum(e_ms), ws)
        # two steps in flight: a second batch of the same scenes and settings on its own
        # stream, each driven by its own host thread (hr_batch_run returns when its step is
        # done), so one batch's uploads and readbacks overlap the other's build and render;
        # every step still uploads all vertices and reads back all images
        import threading
        stream2 = torch.cuda.Stream(device=dev)
        b2 = Batch(dev, stream=stream2.cuda_stream)
        b2.set_scenes(specs)
        b2.set_integrator(0.1, DEFAULT_SEED)
        b2.set_densities(top, leaf)
        if tuning:
            b2.set_launch(tuning["block_threads"], tuning["tile_width"])
        himg2 = torch.zeros(npx * 3, dtype=torch.float32).pin_memory().numpy()
        bs, strs, imgs = [b, b2], [stream, stream2], [himg, himg2]
        errors = []

        def worker(k, nsteps):
            try:
                torch.cuda.set_device(dev)
                for _ in range(nsteps):
                    with torch.cuda.stream(strs[k]):
                        flush.zero_()
                    bs[k].set_vertices(hv)
                    bs[k].run(0)
                    bs[k].download_images(imgs[k])
            except Exception as ex:   # reported after the join
                errors.append(ex)

        def both(nsteps):
            ts = [threading.Thread(target=worker, args=(k, (nsteps + 1 - k) // 2)) for k in range(2)]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            if errors:
                raise errors[0]

        both(max(2, args.warmup))
        torch.cuda.synchronize()
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stream2.wait_event(a)
        both(args.steps)
        stream.wait_stream(stream2)
        z.record(stream)
        z.synchronize()
        et = max_over_ranks(a.elapsed_time(z), ws)
        b2.close()
        e2e = {"value": replica_value(rays_per_step, args.steps, et, ws), "unit": "Mrays/s",
               "h2d_bytes_per_step": int(hv.nbytes), "d2h_bytes_per_step": int(himg.nbytes),
               "ms_per_step": et / args.steps,
               "how": "public C-ABI (hr_batch_set_vertices from pinned host memory, hr_batch_run, "
                      "hr_batch_download_images into pinned memory), two steps in flight on two batches driven by "
                      "two host threads; L2 flushed before every step inside the timed region",
               "one_frame_at_a_time": {"value": replica_value(rays_per_step, args.steps, et_serial, ws),
                                       "ms_per_step": et_serial / args.steps}}

    # the plain per-scene path on the same scenes: one context per scene, all on one
    # stream, each step a build + render of every scene
    engines, fbs = [], []
    for sp in specs:
        e = Engine(dev, stream=stream.cuda_stream)
        e.upload(sp.vertices, sp.vertices, sp.faces, 1.0)
        e.setGridDensities(top, leaf)
        e.setCamera(sp.position, sp.orientation, sp.up, sp.fov, sp.width, sp.height)
        e.set_integrator(ao_samples=sp.ao_samples, ao_radius=-0.1, seed=DEFAULT_SEED)
        engines.append(e)
        fbs.append(torch.zeros(sp.width * sp.height * 3, dtype=torch.float32, device=f"cuda:{dev}"))

    def plain_step():
        for e, fb in zip(engines, fbs):
            e.build(GRID_TWO_LEVEL)
            e.render_device(fb, 0, RENDER_AO)

    # one instrumented pass: ray counts must match the batch; cells / tests size the
    # algorithmic traversal bytes, the grids the algorithmic build bytes
    for e in engines:
        e.set_stats(True)
        e.counters(reset=True)
    plain_step()
    torch.cuda.synchronize()
    st = [e.counters(reset=True) for e in engines]
    plain_rays = sum(s["rays"] for s in st)
    b_trace = sum(trace_bytes(s["rays"], s["cells"], s["tests"]) for s in st)
    b_build = 0
    for e, sp in zip(engines, specs):
        e.set_stats(False)
        b_build += algorithmic_build_bytes(e.grid_info(), sp.vertices.shape[0], sp.faces.shape[0], lerp=False)
    plain_ms = []
    for i in range(args.warmup + max(1, args.steps // 4)):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plain_step()
        z.record(stream)
        z.synchronize()
        if i >= args.warmup:
            plain_ms.append(a.elapsed_time(z))
    for e in engines:
        e.cleanup()
    plain_value = plain_rays / (statistics.median(plain_ms) * 1e-3) / 1e6

    if rank != 0:
        b.close()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    rmed, bmed = statistics.median(render_ms), statistics.median(build_ms)
    ntri = sum(s.faces.shape[0] for s in specs)
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generators, no dataset)",
        "config": {"workload": W["name"], "scenes": len(specs), "triangles": int(ntri),
                   "pixels": int(sum(s.width * s.height for s in specs)), "ao_samples": 4,
                   "densities": [top, leaf], "block_threads": tuning["block_threads"] if tuning else 256,
                   "tile_width": tuning["tile_width"] if tuning else 8, "cuda_graph": True,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{ws}"},
        "rays_per_step": rays_per_step, "build_ms_per_step": bmed, "render_ms_per_step": rmed,
        "plain_path": {"value": plain_value, "unit": "Mrays/s", "ms_per_step": statistics.median(plain_ms),
                       "rays_per_step": plain_rays, "note": "one hr_ctx per scene: build + render each, one stream"},
        "speedup_vs_plain": value / plain_value,
        "autotune": dict(tuning, seconds=tune_s) if tuning else None,
        "roofline": {"bound": "hbm", "kernel": "k_trace_jobs", "achieved": b_trace / (rmed * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": b_trace / (rmed * 1e-3) / 1e9 / peak,
                     "traffic": profile_traffic("k_trace_jobs", W["name"]),
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": b_trace, "kernel_ms": rmed},
        "build_roofline": {"bound": "hbm", "achieved": b_build / (bmed * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": b_build / (bmed * 1e-3) / 1e9 / peak, "algorithmic_bytes": b_build},
        "gpu_launches": launches,
        "e2e": e2e,
    }
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if not args.no_cpu and ws == 1:
        try:
            line["cpu_baseline"] = cpu_baseline_batch(specs, top, leaf)
        except Exception as ex:   # the CPU leg is a reported baseline only
            line["cpu_baseline"] = {"error": str(ex)}
    print(json.dumps(line), flush=True)
    b.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def served_requests(pool, n, rate, seed=0):
    """Poisson arrivals at `rate` req/s; each request draws a scene, a frame time U[0,1) of
    the animation (snapped to its 120 evenly spaced frame times), a square image whose
    pixel count is log-uniform in [128^2, 1024^2], spp in {1, 4, 16} and AO or 4-bounce PT."""
    from happyray_b200 import scenes as S
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for i in range(n):
        sc = int(rng.integers(0, len(pool)))
        kf = pool[sc][0]
        K = kf.shape[0]
        frame = int(rng.uniform(0.0, 1.0) * 120)
        side = int(round(math.sqrt(math.exp(rng.uniform(math.log(128 * 128), math.log(1024 * 1024))))))
        spp = int(rng.choice([1, 4, 16]))
        pt = bool(rng.random() < 0.5)
        reqs.append(dict(at=float(t[i]), scene=sc, ft=K * frame / 120.0, side=side, spp=spp, pt=pt,
                         cam=S.camera_at_bounds(kf[0], (side, side))))
    return reqs


def serve_run(pool, reqs, mode, budget, seed=DEFAULT_SEED):
    """Replays the arrival schedule against one server; returns latency and throughput."""
    import torch
    from happyray_b200 import RENDER_AO, RENDER_PATH
    from happyray_b200.server import Server
    srv = Server(0, budget, mode)
    t0 = time.perf_counter()
    for kf, f in pool:
        srv.add_scene(kf, f)
    load_s = time.perf_counter() - t0
    # pinned result buffers (one allocation), so result copies overlap the next wave
    sizes = [r["side"] * r["side"] * 3 for r in reqs]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    host = torch.empty(int(offs[-1]), dtype=torch.float32).pin_memory().numpy()
    # warm-up (not measured): one small request per integrator
    for r in reqs[:4]:
        cam = dict(r["cam"], res_x=32, res_y=32)
        srv.submit_render(r["scene"], r["ft"], RENDER_PATH if r["pt"] else RENDER_AO, 1, cam, seed).wait()
    s0 = srv.stats()
    pend = []
    start = time.perf_counter()
    for i, r in enumerate(reqs):
        while True:   # open-loop arrivals
            dt = start + r["at"] - time.perf_counter()
            if dt <= 0:
                break
            time.sleep(dt if dt > 2e-3 else 0)
        out = host[offs[i]:offs[i + 1]].reshape(-1, 3)
        pend.append(srv.submit_render(r["scene"], r["ft"], RENDER_PATH if r["pt"] else RENDER_AO, r["spp"],
                                      r["cam"], seed, out=out))
    for p in pend:
        p.wait()
    s1 = srv.stats()
    infos = [p.info() for p in pend]
    srv.close()
    lat = np.array([(i["done_ns"] - i["submit_ns"]) * 1e-6 for i in infos])
    span_s = (max(i["done_ns"] for i in infos) - min(i["submit_ns"] for i in infos)) * 1e-9
    rays = s1["rays"] - s0["rays"]
    return {"mrays_s": rays / span_s / 1e6, "rays": int(rays), "span_s": span_s,
            "completed_per_s": len(reqs) / span_s, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "waves": int(s1["waves"] - s0["waves"]), "rebuilds": int(s1["rebuilds"] - s0["rebuilds"]),
            "failed": int(s1["failed"] - s0["failed"]), "peak_inflight_bytes": int(s1["peak_inflight_bytes"]),
            "resident_bytes": int(s1["resident_bytes"]), "launches": int(s1["launches"] - s0["launches"]),
            "trace_ms": float(s1["trace_ms"] - s0["trace_ms"]),
            "scene_load_s": load_s}


def run_served(args, rank, ws, local):
    """c5: served rendering (continuous batching over resident animated scenes) against
    the plain per-frame path and the serial per-scene path on resident scenes, on one
    replayed Poisson arrival schedule."""
    import torch
    from happyray_b200 import scenes as S
    from happyray_b200.server import BATCHED, PLAIN, SERIAL
    n_req = args.requests
    name = f"c5_served_64_scenes_{n_req}_requests_2000rps"
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the served workload has no CPU form in the "
                              "reference (no server); the CPU baseline of the same integrators is the c2/c3 lines"}),
                  flush=True)
        return
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    pool = S.served_scenes(64, 0, device=f"cuda:{local}")
    gen_s = time.perf_counter() - t0
    reqs = served_requests(pool, n_req, 2000.0)
    budget = 120 << 30
    with ClockSampler(local) as clk:
        served = serve_run(pool, reqs, BATCHED, budget)
        serial = serve_run(pool, reqs, SERIAL, budget)
        plain = serve_run(pool, reqs, PLAIN, budget)
        # latency of continuous batching at loads the server sustains: the same request mix
        # arriving at 50% and 80% of the request rate the server just completed at 2000 req/s
        capacity_rps = served["completed_per_s"]
        at_load = []
        if not args.no_load_sweep:
            for frac in (0.5, 0.8):
                rate = frac * capacity_rps
                n_l = max(50, min(n_req, int(rate * args.load_seconds)))
                lreqs = served_requests(pool, n_l, rate, seed=1)
                r = serve_run(pool, lreqs, BATCHED, budget)
                at_load.append({"offered_fraction_of_capacity": frac, "arrival_rate_rps": rate, "requests": n_l,
                                "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "mean_ms": r["mean_ms"],
                                "mrays_s": r["mrays_s"], "completed_per_s": r["completed_per_s"],
                                "waves": r["waves"]})
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": served["mrays_s"], "unit": "Mrays/s", "n_gpus": ws, "steps": n_req,
        "warmup": 4, "ms_per_step": served["mean_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generators, no dataset)",
        "config": {"workload": name, "scenes": len(pool), "triangles": int(sum(f.shape[0] for _, f in pool)),
                   "keyframes": 16, "arrivals": "Poisson 2000 req/s, open loop", "requests": n_req,
                   "frame_times": "U[0,1) snapped to 120 per cycle", "resolution": "log-uniform 128^2..1024^2",
                   "spp": [1, 4, 16], "integrators": ["AO", "PT 4 bounces"], "hbm_budget_gb": 120,
                   "parallelism": f"replicas x{ws}"},
        "served": served,
        "plain_path": dict(plain, note="the drop-in per-frame path: one context; per request upload the two key "
                                      "frames around the frame time, build, render, read back"),
        "serial_resident_path": dict(serial, note="per-scene path one request at a time on the resident scenes "
                                                  "(no batching, no overlap)"),
        "speedup_vs_plain": served["mrays_s"] / plain["mrays_s"],
        "speedup_vs_serial_resident": served["mrays_s"] / serial["mrays_s"],
        "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
        "capacity_rps": capacity_rps,
        "latency_at_sustained_load": at_load,
        "timing": "wall clock from each request's submission to its completion (results in pinned host memory); "
                  "throughput = rays / (last completion - first submission)",
        "scene_generation_s": gen_s,
        "gpu_launches": served["launches"],
        "e2e": {"value": served["mrays_s"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(r["side"] ** 2 * 12 for r in reqs) / n_req),
                "note": "every request is end to end: submission to result in host memory"},
    }
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    print(json.dumps(line), flush=True)


def hier_workload(seed: int = 0, frames: int = 8):
    """Instanced hierarchy workload: 64 objects (icospheres and heightfield tiles, 320-20480
    triangles) x 16,384 rigid instances (scales 0.01-0.05 in [0, 1]^3), 8 rigid-body frames
    (every instance shifted by a seeded offset per frame), 1920x1080 pinhole rays at the
    instance bounds listed in 8x4 pixel tiles, object / instance densities 1.2 / 1.2
    (RTEngine.cu:72-73)."""
    from happyray_b200 import scenes as S
    v, f, counts, inst = S.instanced_scene(64, 16384, seed=seed, tri_range=(320, 20480), world=1.0,
                                           scale_range=(0.01, 0.05))
    rng = np.random.default_rng(seed + 1)
    seq = []
    for k in range(frames):
        m = inst.copy()
        shift = (rng.normal(0, 0.01, (len(inst), 3)) * k).astype(np.float32)
        m["bmin"] += shift
        m["bmax"] += shift
        mm = m["m"].reshape(-1, 3, 4).astype(np.float64)
        mm[:, :, 3] -= np.einsum("nij,nj->ni", mm[:, :, :3], shift.astype(np.float64))
        m["m"] = mm.reshape(-1, 12).astype(np.float32)
        seq.append(m)
    W, H = 1920, 1080
    lo, hi = inst["bmin"].min(0).astype(np.float64), inst["bmax"].max(0).astype(np.float64)
    c = 0.5 * (lo + hi)
    pos = np.array([0.5, -0.8, 0.9]) * (hi - lo) + lo
    fwd = (c - pos) / np.linalg.norm(c - pos)
    right = np.cross(fwd, [0.0, 0.0, 1.0]); right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    th = math.tan(math.radians(60.0) / 2)
    xs = ((np.arange(W) + 0.5) / W * 2 - 1) * th * W / H
    ys = (1 - (np.arange(H) + 0.5) / H * 2) * th
    d = fwd[None, None, :] + xs[None, :, None] * right[None, None, :] + ys[:, None, None] * up[None, None, :]
    d = (d / np.linalg.norm(d, axis=2, keepdims=True)).astype(np.float32)
    # the rays in 8x4 pixel tiles (as the library's camera kernels issue them), so that the
    # 32 rays of a warp start into a small solid angle
    d = np.ascontiguousarray(d.reshape(H // 4, 4, W // 8, 8, 3).transpose(0, 2, 1, 3, 4)).reshape(-1, 3)
    org = np.broadcast_to(pos.astype(np.float32), d.shape).copy()
    return dict(name="c6_instanced_hierarchy_64_objects_16384_instances_1080p", v=v, f=f, counts=counts,
                frames=seq, org=org, dir=d, res=(W, H))


def hier_bytes(rays, st):
    """Algorithmic traversal bytes of the hierarchy: per ray 24 B ray + 20 B hit, 8 B per
    instance-grid cell, 80 B per instance record tested, 72 B per object record of an
    entered instance, 8 B per object-grid cell, 52 B per triangle test."""
    s = st.sum(axis=0).astype(np.float64)
    return 44.0 * rays + 8 * s[0] + 80 * s[1] + 72 * s[2] + 8 * s[3] + 52 * s[4]


def cpu_baseline_hier(W, stride=16):
    import oracle as O
    t0 = time.perf_counter()
    ob = O.hier_build(W["v"], W["f"], W["counts"], W["frames"][0], 1.2, 1.2)
    tb = time.perf_counter() - t0
    org, d = W["org"][::stride], W["dir"][::stride]
    t0 = time.perf_counter()
    O.hier_trace(ob, org, d)
    tt = time.perf_counter() - t0
    n = W["org"].shape[0]
    return {"value": n / (tb + tt * stride) / 1e6, "unit": "Mrays/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"full build ({tb * 1e3:.0f} ms) + every {stride}th ray ({org.shape[0]} rays, "
                      f"{tt * 1e3:.0f} ms) scaled to the full frame", "build_ms": tb * 1e3}


def run_hier(args, rank, ws, local):
    """c6: the instanced two-level grid hierarchy, one rigid-body frame per step: the
    frame's instances to the device, the instance grid rebuilt, 1080p primary rays traced
    (closest hit) through instance grid and object grids."""
    W = hier_workload()
    n = W["org"].shape[0]
    if args.impl == "reference":
        if rank == 0:
            vals = [cpu_baseline_hier(W) for _ in range(max(1, args.steps // 10))]
            cb = vals[-1]
            v = statistics.median(x["value"] for x in vals)
            print(json.dumps({"metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": 1, "steps": len(vals),
                              "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f32", "data": "synthetic (seeded)", "config": {"workload": W["name"]},
                              "impl": "reference", "cpu_baseline": dict(cb, value=v),
                              "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    from happyray_b200.hier import Hierarchy
    dev = local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    h = Hierarchy(dev, stream.cuda_stream)
    t0 = time.perf_counter()
    h.set_objects(W["v"], W["f"], W["counts"])
    h.set_instances(W["frames"][0])
    h.build()
    full_build_s = time.perf_counter() - t0
    dorg = torch.from_numpy(W["org"]).to(f"cuda:{dev}")
    ddir = torch.from_numpy(W["dir"]).to(f"cuda:{dev}")
    outs = [torch.empty(n, dtype=torch.int32, device=f"cuda:{dev}"), torch.empty(n, dtype=torch.int32, device=f"cuda:{dev}")]
    outs += [torch.empty(n, dtype=torch.float32, device=f"cuda:{dev}") for _ in range(3)]
    stats = torch.empty((n, 5), dtype=torch.int32, device=f"cuda:{dev}")
    h.trace_stats_device(dorg, ddir, *outs, stats)
    torch.cuda.synchronize()
    st = stats.cpu().numpy().astype(np.int64)
    b_trace = hier_bytes(n, st)
    hit_frac = float((outs[0] >= 0).float().mean())
    K = len(W["frames"])

    def step(i, evs=None):
        if evs:
            evs[0].record(stream)
        h.set_instances(W["frames"][i % K])
        h.build()
        if evs:
            evs[1].record(stream)
        h.trace_rays_device(dorg, ddir, *outs)
        if evs:
            evs[2].record(stream)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    l0 = h.info()["launches"]
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    with ClockSampler(dev) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            step(i, evs[i])
        torch.cuda.synchronize()
    launches = h.info()["launches"] - l0
    build_ms = [e[0].elapsed_time(e[1]) for e in evs]
    trace_ms = [e[1].elapsed_time(e[2]) for e in evs]
    total_ms = max_over_ranks(sum(b + t for b, t in zip(build_ms, trace_ms)), ws)
    value = replica_value(n, args.steps, total_ms, ws)
    e2e = None
    if not args.no_e2e:
        horg = torch.from_numpy(W["org"]).pin_memory().numpy()
        hdir = torch.from_numpy(W["dir"]).pin_memory().numpy()
        # the hits land in page-locked host buffers (allocated once)
        hout = [torch.empty(n, dtype=dt).pin_memory().numpy()
                for dt in (torch.int32, torch.int32, torch.float32, torch.float32, torch.float32)]
        e_ms = []
        for i in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            h.set_instances(W["frames"][i % K])
            h.build()
            res = h.trace_rays(horg, hdir, out=hout)
            z.record(stream)
            z.synchronize()
            if i >= args.warmup:
                e_ms.append(a.elapsed_time(z))
        et_serial = max_over_ranks(sum(e_ms), ws)
        # two frames in flight, as in the per-scene lines: frame i on hierarchy i % 2 (own
        # stream, device and pinned buffers); each frame uploads its instances (set_instances
        # and build wait only for their own hierarchy's stream) and its rays, traces, and
        # reads its hits back, while the other hierarchy's frame runs
        stream2 = torch.cuda.Stream(device=dev)
        h2 = Hierarchy(dev, stream2.cuda_stream)
        h2.set_objects(W["v"], W["f"], W["counts"])
        h2.set_instances(W["frames"][0])
        h2.build()
        hs, strs = [h, h2], [stream, stream2]
        horg_t, hdir_t = torch.from_numpy(horg), torch.from_numpy(hdir)
        dev_bufs, pin_bufs = [], []
        for k in range(2):
            rays = (torch.empty((n, 3), dtype=torch.float32, device=f"cuda:{dev}"),
                    torch.empty((n, 3), dtype=torch.float32, device=f"cuda:{dev}"))
            hits = [torch.empty(n, dtype=dt, device=f"cuda:{dev}")
                    for dt in (torch.int32, torch.int32, torch.float32, torch.float32, torch.float32)]
            dev_bufs.append((rays, hits))
            pin_bufs.append([torch.empty(n, dtype=x.dtype).pin_memory() for x in hits])

        def frame(i):
            k = i % 2
            (dorg_k, ddir_k), hits = dev_bufs[k]
            with torch.cuda.stream(strs[k]):
                flush.zero_()
            hs[k].set_instances(W["frames"][i % K])
            hs[k].build()
            with torch.cuda.stream(strs[k]):
                dorg_k.copy_(horg_t, non_blocking=True)
                ddir_k.copy_(hdir_t, non_blocking=True)
            hs[k].trace_rays_device(dorg_k, ddir_k, *hits)
            with torch.cuda.stream(strs[k]):
                for hb, db in zip(pin_bufs[k], hits):
                    hb.copy_(db, non_blocking=True)

        for i in range(args.warmup):
            frame(i)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stream2.wait_event(a)
        for i in range(args.steps):
            frame(args.warmup + i)
        stream.wait_stream(stream2)
        b.record(stream)
        b.synchronize()
        et = max_over_ranks(a.elapsed_time(b), ws)
        h2.close()
        e2e = {"value": replica_value(n, args.steps, et, ws), "unit": "Mrays/s",
               "h2d_bytes_per_step": int(horg.nbytes + hdir.nbytes + W["frames"][0].nbytes),
               "d2h_bytes_per_step": int(sum(x.nbytes for x in hout)), "ms_per_step": et / args.steps,
               "how": "public C-ABI (hr_hier_set_instances, hr_hier_build, rays copied from pinned host memory, "
                      "hr_hier_trace_rays_device, hits read back into pinned memory), two frames in flight on two "
                      "hierarchies; L2 flushed before every frame inside the timed region",
               "one_frame_at_a_time": {"value": replica_value(n, args.steps, et_serial, ws),
                                       "ms_per_step": et_serial / args.steps,
                                       "how": "hr_hier_set_instances, hr_hier_build, hr_hier_trace_rays (host rays "
                                              "in, hits into pinned host buffers), one frame after the other"}}
    if rank != 0:
        h.close()
        return
    peak, peak_kind = peaks()
    tmed, bmed = statistics.median(trace_ms), statistics.median(build_ms)
    info = h.info()
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generators, no dataset)",
        "config": {"workload": W["name"], "objects": int(len(W["counts"])), "triangles": int(W["f"].shape[0]),
                   "instances": int(len(W["frames"][0])),
                   "instanced_triangles": int(W["counts"][W["frames"][0]["obj"]].sum()),
                   "resolution": list(W["res"]), "densities": [1.2, 1.2], "rigid_frames": K,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{ws}"},
        "rays_per_step": n, "hit_fraction": hit_frac,
        "instance_rebuild_ms_per_frame": bmed, "trace_ms_per_frame": tmed, "full_build_s_first": full_build_s,
        "grid": info,
        "per_ray": {k: float(st[:, j].mean()) for j, k in enumerate(
            ["instance_grid_cells", "instance_boxes_tested", "instances_entered", "object_grid_cells",
             "triangle_tests"])},
        "roofline": {"bound": "hbm", "kernel": "k_hier_trace", "achieved": b_trace / (tmed * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": b_trace / (tmed * 1e-3) / 1e9 / peak,
                     "traffic": profile_traffic("k_hier_trace", W["name"]),
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": b_trace, "kernel_ms": tmed},
        "gpu_launches": launches,
        "e2e": e2e,
    }
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if not args.no_cpu and ws == 1:
        try:
            line["cpu_baseline"] = cpu_baseline_hier(W)
        except Exception as ex:   # the CPU leg is a reported baseline only
            line["cpu_baseline"] = {"error": str(ex)}
    print(json.dumps(line), flush=True)
    h.close()


def configure(eng, W, frames):
    """The workload's mesh, grid settings, camera, integrator and light on an Engine."""
    cam = W["cam"]
    eng.set_keyframes(frames, W["f"])
    if W["kind"] == 0:
        eng.set_uniform_density(W["ug"])
    else:
        eng.setGridDensities(W["top"], W["leaf"])
    eng.setCamera(cam["position"], cam["orientation"], cam["up"], cam["fov"], cam["res_x"], cam["res_y"])
    if W["mode"] == 3:
        eng.set_integrator(ao_samples=W["ao"], ao_radius=-0.1)
    elif W["mode"] == 1:
        eng.set_integrator(pt_bounces=W["bounces"], albedo=0.7)
        eng.setLights((0.4, 0.4, 1.0), (0.2, 0.0, 0.0), (0.0, 0.2, 0.0), 20.0)


def fast_arith_leg(args, W, dev, stream, frames, flush, times_fn, keep, ieee_value):
    """The same frames through libhappyray_b200_fast.so (traversal kernels with FMA
    contraction and approximate division; the grid build is the IEEE one), timed like the
    main steps, and its output on the CPU baseline's frame compared with the oracle's."""
    import torch
    from happyray_b200 import Engine, _lib
    fe = Engine(dev, stream=stream.cuda_stream, lib=_lib.load_fast())
    try:
        configure(fe, W, frames)
        npx = W["cam"]["res_x"] * W["cam"]["res_y"]
        fb = torch.zeros(npx * 3, dtype=torch.float32, device=f"cuda:{dev}")

        def step(i, evs=None):
            fe.set_frame_time(times_fn(i), 0.0)
            if evs:
                evs[0].record(stream)
            fe.build(W["kind"], W.get("exact", True))
            fe.render_device(fb, 0, W["mode"])
            if evs:
                evs[1].record(stream)

        fe.set_stats(True)
        fe.counters(reset=True)
        step(0)
        fe.sync()
        rays = fe.counters(reset=True)["rays"]
        fe.set_stats(False)
        for i in range(args.warmup):
            step(i)
        fe.sync()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            step(args.warmup + i, evs[i])
        fe.sync()
        torch.cuda.synchronize()
        ms = sum(e[0].elapsed_time(e[1]) for e in evs)
        value = rays * args.steps / (ms * 1e-3) / 1e6
        out = {"library": "libhappyray_b200_fast.so", "value": value, "unit": "Mrays/s",
               "ms_per_step": ms / args.steps, "vs_ieee_build": value / ieee_value if ieee_value else None,
               "rays_per_step": rays}
        if keep and W["mode"] in (1, 3):
            f1, f2, coeff = baseline_frame(W)
            fe.upload(f1, f2, W["f"], coeff)
            fe.build(W["kind"], W.get("exact", True))
            gi, cells, leaves, prims = fe.grid_download()
            b = keep["grid"]
            grid_equal = bool(np.array_equal(cells, b.cells) and np.array_equal(prims, b.prims) and
                              (b.leaves is None or np.array_equal(leaves, b.leaves)))
            fe.render_device(fb, 0, W["mode"])
            fe.sync()
            st = keep["stride"]
            img = fb.view(-1, 3).cpu().numpy()[::st, 0].astype(np.float64)
            ref = np.asarray(keep["out"])[::st].astype(np.float64)
            d = np.abs(img - ref)
            out["vs_oracle"] = {"grid_bit_exact": grid_equal, "pixels_compared": int(d.size),
                                "pixels_differing": int((d > 0).sum()), "max_abs_diff": float(d.max()),
                                "rmse": float(np.sqrt((d * d).mean())),
                                "image_range": [float(ref.min()), float(ref.max())]}
        return out
    finally:
        fe.cleanup()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "c6"])
    ap.add_argument("--requests", type=int, default=1000, help="c5: requests replayed per mode")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="c4: skip the autotuner (densities 1/16, 2)")
    ap.add_argument("--no-rebuild2m", action="store_true", help="c2: skip the 2M-triangle key-frame rebuild")
    ap.add_argument("--no-fast", action="store_true", help="c2/c3: skip the fast-arithmetic build's leg")
    ap.add_argument("--no-load-sweep", action="store_true", help="c5: skip the latency runs at sustained loads")
    ap.add_argument("--load-seconds", type=float, default=6.0, help="c5: arrival span of each sustained-load run")
    args = ap.parse_args()
    rank, ws, local = dist_setup() if os.environ.get("WORLD_SIZE") else (0, 1, 0)
    if args.config == "c4":
        run_batched(args, rank, ws, local)
        return
    if args.config == "c5":
        run_served(args, rank, ws, local)
        return
    if args.config == "c6":
        run_hier(args, rank, ws, local)
        return

    W = workload(args.config)
    if args.impl == "reference":
        run_reference(args, W, rank, ws)
        return

    import torch
    from happyray_b200 import Engine
    dev = local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    eng = Engine(dev, stream=stream.cuda_stream)
    v, f, cam = W["v"], W["f"], W["cam"]
    frames = W["frames"]
    if frames is None:
        frames = v[None]
    configure(eng, W, frames)
    npx = cam["res_x"] * cam["res_y"]
    d_fb = torch.zeros(npx * 3, dtype=torch.float32, device=f"cuda:{dev}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    K = frames.shape[0]
    times = [16.0 * k / 120.0 for k in range(120)] if K > 1 else [0.0]

    def frame_time(i):
        t = times[i % len(times)]
        return t if K > 1 else 0.0

    def step(i, evs=None):
        eng.set_frame_time(frame_time(i), 0.0)
        if evs:
            evs[0].record(stream)
        eng.build(W["kind"], W.get("exact", True))
        if evs:
            evs[1].record(stream)
        eng.render_device(d_fb, 0, W["mode"])
        if evs:
            evs[2].record(stream)

    # algorithmic figures from an instrumented frame (not timed)
    eng.set_stats(True)
    eng.counters(reset=True)
    step(0)
    eng.sync()
    st = eng.counters(reset=True)
    eng.set_stats(False)
    gi = eng.grid_info()
    rays_per_step = st["rays"]
    # algorithmic bytes of each render kernel: primary pass, secondary pass (AO samples)
    b_primary = trace_bytes(st["rays"] - st["rays2"], st["cells"] - st["cells2"], st["tests"] - st["tests2"])
    b_secondary = trace_bytes(st["rays2"], st["cells2"], st["tests2"])
    b_build = algorithmic_build_bytes(gi, v.shape[0], f.shape[0], lerp=True)
    eng.set_timing(True)

    for i in range(args.warmup):
        step(i)
    eng.sync()
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    prep2m = rebuild_2m_prepare(dev, stream) if args.config == "c2" and not args.no_rebuild2m else None
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    l0 = eng.counters()["launches"]
    kern_ms = []
    clk = ClockSampler(dev)
    clk.__enter__()   # sampled over every timed region below (steps, end to end, 2M rebuild)
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()   # L2 flush between timed steps (256 MiB > 126 MB L2), outside the events
        step(args.warmup + i, evs[i])
        kern_ms.append(eng.render_times())
    eng.sync()
    torch.cuda.synchronize()
    launches = eng.counters()["launches"] - l0
    build_ms = [e[0].elapsed_time(e[1]) for e in evs]
    trace_ms = [e[1].elapsed_time(e[2]) for e in evs]
    step_ms = [b + t for b, t in zip(build_ms, trace_ms)]
    total_ms = max_over_ranks(sum(step_ms), ws)
    value = replica_value(rays_per_step, args.steps, total_ms, ws)

    # end to end through the public API: pinned host inputs, upload + build + render + readback
    e2e = None
    if not args.no_e2e:
        hv = torch.from_numpy(np.ascontiguousarray(frames[0])).pin_memory().numpy()
        hf = torch.from_numpy(f.view(np.int32)).pin_memory().numpy().view(np.uint32)
        hfb = torch.zeros((npx, 3), dtype=torch.float32).pin_memory().numpy()
        # one frame at a time: upload, build, render into the host frame buffer, wait
        e_ms = []
        for i in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            eng.upload(hv, hv, hf, 1.0)
            eng.build(W["kind"], W.get("exact", True))
            eng.renderFrame(hfb, 0, W["mode"])
            b.record(stream)
            b.synchronize()
            if i >= args.warmup:
                e_ms.append(a.elapsed_time(b))
        et_serial = max_over_ranks(sum(e_ms), ws)
        # two frames in flight: frame i on context i % 2 (own stream, own device and pinned
        # frame buffers), so one frame's readback and the next one's upload overlap the other
        # context's build and render; every frame still uploads its inputs and reads back
        # its image, inside one timed region around all frames
        stream2 = torch.cuda.Stream(device=dev)
        eng2 = Engine(dev, stream=stream2.cuda_stream)
        configure(eng2, W, frames)
        engs, strs = [eng, eng2], [stream, stream2]
        d_fbs = [d_fb, torch.zeros_like(d_fb)]
        h_fbs = [torch.zeros(npx * 3, dtype=torch.float32).pin_memory() for _ in range(2)]

        def frame(i):
            k = i % 2
            with torch.cuda.stream(strs[k]):
                flush.zero_()
            engs[k].upload(hv, hv, hf, 1.0)
            engs[k].build(W["kind"], W.get("exact", True))
            engs[k].render_device(d_fbs[k], 0, W["mode"])
            with torch.cuda.stream(strs[k]):
                h_fbs[k].copy_(d_fbs[k], non_blocking=True)

        for i in range(args.warmup):
            frame(i)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stream2.wait_event(a)
        for i in range(args.steps):
            frame(args.warmup + i)
        stream.wait_stream(stream2)
        b.record(stream)
        b.synchronize()
        et = max_over_ranks(a.elapsed_time(b), ws)
        eng2.cleanup()
        e2e = {"value": replica_value(rays_per_step, args.steps, et, ws), "unit": "Mrays/s",
               "h2d_bytes_per_step": int(2 * hv.nbytes + hf.nbytes), "d2h_bytes_per_step": int(hfb.nbytes),
               "ms_per_step": et / args.steps,
               "how": "public C-ABI (hr_upload, hr_build, hr_render_device, then a pinned readback), two frames in "
                      "flight on two contexts; L2 flushed before every frame inside the timed region",
               "one_frame_at_a_time": {"value": replica_value(rays_per_step, args.steps, et_serial, ws),
                                       "ms_per_step": et_serial / args.steps}}
    # the headline line also carries the 2M-triangle key-frame rebuild (replayed build graph)
    rebuild2m = None
    if prep2m is not None:
        rb_ms, rb_bytes, rb_n = rebuild_2m_keyframe(prep2m, stream, flush)
        prep2m[0].cleanup()
        rb_ms = max_over_ranks(rb_ms, ws)
        rebuild2m = {"ms": rb_ms, "frame_times": rb_n, "algorithmic_bytes": rb_bytes,
                     "achieved_gbs": rb_bytes / (rb_ms * 1e-3) / 1e9}
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)

    if rank != 0:
        eng.cleanup()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    l2_peak = l2_read_gbs(stream)
    tl = W["kind"] == 1   # two-level AO kernels refill lanes inside the traversal loop
    ao = ["k_ao_primary_tl" if tl else "k_ao_primary", "k_ao_samples_tl" if tl else "k_ao_samples", "k_ao_finish"]
    names = {0: ["k_render_primary"], 1: ["k_render_pt"], 3: ao}[W["mode"]]
    kbytes = {0: [b_primary + b_secondary], 1: [b_primary + b_secondary], 3: [b_primary, b_secondary, 0]}[W["mode"]]
    kmed = [statistics.median(k[j] for k in kern_ms) for j in range(len(names))] if kern_ms and kern_ms[0] else [0.0]
    top = max(range(len(kmed)), key=lambda j: kmed[j])
    kern = names[top]
    b_trace = kbytes[top]
    tr_med = statistics.median(trace_ms)
    achieved = b_trace / (kmed[top] * 1e-3) / 1e9 if kmed[top] > 0 else 0.0
    traffic = profile_traffic(kern, W["name"])
    bmed = statistics.median(build_ms)
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generators, no dataset)",
        "config": {"workload": W["name"], "triangles": int(f.shape[0]), "vertices": int(v.shape[0]),
                   "resolution": [cam["res_x"], cam["res_y"]], "grid": "two-level" if W["kind"] else "uniform",
                   "densities": [W.get("top", W.get("ug")), W.get("leaf")], "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas x{ws}"},
        "rays_per_step": rays_per_step, "build_ms_per_frame": bmed, "trace_ms_per_frame": tr_med,
        "trace_mrays_s": rays_per_step / (tr_med * 1e-3) / 1e6,
        "grid": {k: gi[k] for k in ("res", "num_cells", "num_leaves", "num_pairs", "num_top_pairs")},
        "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": b_trace, "kernel_ms": kmed[top],
                     "render_kernels_ms": dict(zip(names, kmed)),
                     "l2": {"peak": l2_peak, "unit": "GB/s", "frac": achieved / l2_peak if l2_peak else None,
                            "how": "L2-resident read rate of this device, measured in this run (hr_probe_l2_read)"}},
        "build_roofline": {"bound": "hbm", "achieved": b_build / (bmed * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": b_build / (bmed * 1e-3) / 1e9 / peak, "algorithmic_bytes": b_build},
        "gpu_launches": launches,
        "e2e": e2e,
    }
    if rebuild2m:
        rebuild2m["hbm_frac"] = rebuild2m["achieved_gbs"] / peak
        line["rebuild_2M_keyframe_ms"] = rebuild2m["ms"]
        line["rebuild_2M_keyframe"] = dict(rebuild2m, workload="c3 mesh: 2,097,152 triangles, 16 curl-noise key "
                                           "frames, two-level 1/16 : 2, key-frame interpolation fused, one "
                                           "replayed build graph per frame time, L2 flushed before each")
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if not args.no_cpu and ws == 1:
        try:
            keep = {}
            line["cpu_baseline"] = cpu_baseline(W, keep=keep)
            line["cpu_baseline"].pop("build_ms", None)
            line["parity"] = gpu_parity(eng, W, keep, d_fb)
        except Exception as ex:   # the CPU leg is a reported baseline only
            line["cpu_baseline"] = {"error": str(ex)}
    if W["mode"] in (1, 3) and ws == 1 and not args.no_fast:
        try:
            line["fast_arith"] = fast_arith_leg(args, W, dev, stream, frames, flush, frame_time,
                                                keep if not args.no_cpu and "grid" in keep else None, value)
        except Exception as ex:   # an extra measurement; the line above stands without it
            line["fast_arith"] = {"error": str(ex)}
    print(json.dumps(line), flush=True)
    eng.cleanup()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
