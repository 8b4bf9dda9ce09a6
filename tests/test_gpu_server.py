"""Served rendering (hr_server_*): every request's result is the same alone, in a mix of
concurrent requests, in serial mode (the per-scene path) and through the plain Engine
calls that render it -- bit-identical, since the result depends only on the request."""
import threading

import numpy as np
import pytest

from happyray_b200 import GRID_TWO_LEVEL, RENDER_AO, RENDER_PATH, RENDER_PRIMARY, Engine, HRError
from happyray_b200 import scenes as S
from happyray_b200.server import BATCHED, PLAIN, SERIAL, Server

pytestmark = pytest.mark.gpu

SEED = 77


def animated(kind, n, seed, nkf=4):
    if kind == "clusters":
        v, f = S.clusters(n, seed)
    else:
        v, f = S.heightfield_tris(n, seed)
    return S.curl_keyframes(v, nkf, amp=0.02, octaves=2, seed=seed), f


@pytest.fixture(scope="module")
def pool():
    return [animated("clusters", 20_000, 1), animated("heightfield", 8_000, 2), animated("clusters", 3_000, 3)]


def requests(pool, n=40, seed=0):
    """A seeded mix: AO (1/4 spp), path (1/2 spp), primary and ray queries."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        sc = int(rng.integers(0, len(pool)))
        kf, _ = pool[sc]
        ft = float(kf.shape[0] * int(rng.integers(0, 8)) / 8.0)
        kind = ["ao", "pt", "primary", "rays"][i % 4]
        side = int(rng.integers(12, 48))
        cam = S.camera_at_bounds(kf[0], (side, side + 3))
        if kind == "rays":
            nr = int(rng.integers(50, 400))
            org = np.tile(np.asarray(cam["position"], np.float32), (nr, 1))
            d = rng.normal(size=(nr, 3)).astype(np.float32) * 0.3 + np.asarray(cam["orientation"], np.float32)
            out.append(dict(kind=kind, scene=sc, ft=ft, org=org, dir=d))
        else:
            spp = {"ao": [1, 4][i % 2], "pt": [1, 2][(i // 4) % 2], "primary": 1}[kind]
            mode = {"ao": RENDER_AO, "pt": RENDER_PATH, "primary": RENDER_PRIMARY}[kind]
            out.append(dict(kind=kind, scene=sc, ft=ft, mode=mode, spp=spp, cam=cam))
    return out


def submit(srv, q):
    if q["kind"] == "rays":
        return srv.submit_rays(q["scene"], q["ft"], q["org"], q["dir"])
    return srv.submit_render(q["scene"], q["ft"], q["mode"], q["spp"], q["cam"], SEED)


def same(a, b):
    if isinstance(a, tuple):
        return all(np.array_equal(x, y) for x, y in zip(a, b))
    return np.array_equal(a, b)


def make_server(pool, mode, budget=8 << 30):
    srv = Server(0, budget, mode)
    for kf, f in pool:
        srv.add_scene(kf, f)
    return srv


@pytest.fixture(scope="module")
def served(hrlib, pool):
    """Results of the mix in batched mode (all submitted at once), serial and plain modes."""
    qs = requests(pool)
    with make_server(pool, BATCHED) as srv:
        pend = [submit(srv, q) for q in qs]
        mix = [p.wait(60_000) for p in pend]
        infos = [p.info() for p in pend]
        st = srv.stats()
    with make_server(pool, SERIAL) as srv:
        ser = [submit(srv, q).wait(60_000) for q in qs]
    with make_server(pool, PLAIN) as srv:
        pla = [submit(srv, q).wait(60_000) for q in qs]
    return qs, mix, ser, infos, st, pla


def test_served_mix_equals_serial_and_plain(served):
    qs, mix, ser, infos, st, pla = served
    for i, (a, b, c) in enumerate(zip(mix, ser, pla)):
        assert same(a, b), f"request {i} ({qs[i]['kind']}) serial"
        assert same(a, c), f"request {i} ({qs[i]['kind']}) plain"
    assert st["completed"] == len(qs) and st["failed"] == 0
    assert all(i["status"] == 2 and i["done_ns"] >= i["submit_ns"] for i in infos)
    # the mix was batched: fewer waves than requests
    assert st["waves"] < len(qs)


def test_served_alone_equals_mix(served, pool):
    qs, mix, _, _, _, _ = served
    with make_server(pool, BATCHED) as srv:
        for i in range(0, len(qs), 5):
            assert same(submit(srv, qs[i]).wait(60_000), mix[i]), f"request {i}"


def test_served_equals_plain_engine(served, pool):
    qs, mix, _, _, _, _ = served
    for i in range(8):
        q = qs[i]
        kf, f = pool[q["scene"]]
        e = Engine(0)
        try:
            e.set_keyframes(kf, f)
            e.set_frame_time(q["ft"], 0.0)
            e.setGridDensities(0.0625, 2.0)
            e.build(GRID_TWO_LEVEL)
            if q["kind"] == "rays":
                ref = e.trace_rays(q["org"], q["dir"])
            else:
                c = q["cam"]
                e.setCamera(c["position"], c["orientation"], c["up"], c["fov"], c["res_x"], c["res_y"])
                e.set_integrator(ao_samples=q["spp"], ao_radius=-0.1, pt_bounces=4, albedo=0.7, seed=SEED)
                ref = None
                if q["mode"] == RENDER_PATH:
                    for k in range(q["spp"]):
                        ref = e.renderFrame(ref, k, RENDER_PATH)
                else:
                    ref = e.renderFrame(None, 0, q["mode"])
            assert same(mix[i], ref), f"request {i} ({q['kind']})"
        finally:
            e.cleanup()


def test_rebuild_only_on_new_frame_time(hrlib, pool):
    cam = S.camera_at_bounds(pool[0][0][0], (16, 16))
    with make_server(pool, BATCHED) as srv:
        base = srv.stats()["rebuilds"]
        for _ in range(3):
            srv.submit_render(0, 1.0, RENDER_AO, 1, cam, SEED).wait(30_000)
        assert srv.stats()["rebuilds"] - base == 1
        srv.submit_render(0, 2.5, RENDER_AO, 1, cam, SEED).wait(30_000)
        assert srv.stats()["rebuilds"] - base == 2


def test_concurrent_submitters(hrlib, pool):
    qs = requests(pool, 24, seed=5)
    with make_server(pool, BATCHED) as srv:
        ref = [submit(srv, q).wait(60_000) for q in qs]
        got = [None] * len(qs)

        def run(k):
            for i in range(k, len(qs), 3):
                got[i] = submit(srv, qs[i]).wait(60_000)

        th = [threading.Thread(target=run, args=(k,)) for k in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for i in range(len(qs)):
            assert same(got[i], ref[i]), f"request {i}"


def test_budget(hrlib, pool):
    kf, f = pool[0]
    with Server(0, 1 << 20, BATCHED) as srv:   # 1 MiB: the scene does not fit
        with pytest.raises(HRError) as ei:
            srv.add_scene(kf, f)
        assert ei.value.status == 2
    with make_server(pool[:1], BATCHED, budget=64 << 20) as srv:
        big = S.camera_at_bounds(kf[0], (4096, 4096))   # 192 MiB of framebuffer > 64 MiB budget
        p = srv.submit_render(0, 0.0, RENDER_AO, 1, big, SEED)
        with pytest.raises(HRError) as ei:
            p.wait(30_000)
        assert ei.value.status == 2
        # the server keeps serving
        small = S.camera_at_bounds(kf[0], (16, 16))
        srv.submit_render(0, 0.0, RENDER_AO, 1, small, SEED).wait(30_000)


def test_invalid_requests(hrlib, pool):
    with make_server(pool[:1], BATCHED) as srv:
        cam = S.camera_at_bounds(pool[0][0][0], (16, 16))
        with pytest.raises(HRError):
            srv.submit_render(5, 0.0, RENDER_AO, 1, cam, SEED)       # unknown scene
        with pytest.raises(HRError):
            srv.submit_render(0, 99.0, RENDER_AO, 1, cam, SEED)      # beyond the key frames
        with pytest.raises(HRError):
            srv.submit_render(0, 0.0, RENDER_AO, 0, cam, SEED)       # no samples


def test_watchdog_answers_a_stuck_wave_and_keeps_serving(hrlib, pool):
    """A wave whose GPU work has not finished within the watchdog's limit is declared stuck
    and its requests fail with HR_ERR_TIMEOUT instead of leaving their callers waiting; the
    server keeps serving.  The stuck wave is made on the host (the worker holds it back:
    hr_server_inject_stall), no GPU work is stalled."""
    cam = S.camera_at_bounds(pool[0][0][0], (24, 24))
    with make_server(pool, BATCHED) as srv:
        ref = srv.submit_render(0, 1.0, RENDER_AO, 2, cam, SEED).wait(30_000)
        srv.set_watchdog(150)
        srv.inject_stall(1, 1500)
        stuck = srv.submit_render(1, 0.5, RENDER_AO, 2, cam, SEED)
        with pytest.raises(HRError) as ei:
            stuck.wait(30_000)
        assert ei.value.status == 5   # HR_ERR_TIMEOUT
        assert srv.stats()["watchdog_trips"] == 1
        # later requests are served (after the held-back wave ends), with the same results
        again = srv.submit_render(0, 1.0, RENDER_AO, 2, cam, SEED).wait(30_000)
        assert same(again, ref)
        srv.drain(30_000)
        assert srv.stats()["watchdog_trips"] == 1
