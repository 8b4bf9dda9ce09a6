"""Seeded synthetic scenes with the shapes of the benchmark configurations.

The reference's sample scenes are not available, so seeded stand-ins are generated:
  * heightfield(): 129x129 vertices over [0,1]^2, height = sum of 4 seeded sinusoids
    (frequency U[1,8], amplitude 0.025 each), 2 triangles per quad (32,768 triangles);
  * clusters(): level-4 icospheres (5,120 triangles each, radius lognormal(ln 0.01, 0.7))
    with centres Gaussian (sigma 0.05) around 64 cluster means uniform in the unit cube,
    plus a 2-triangle ground plane z = 0 over [-0.5, 1.5]^2; the last sphere is truncated
    so the triangle total is exact;
  * curl_keyframes(): per-vertex displacement by a seeded divergence-free (curl) noise
    field, amplitude 0.02, 4 octaves, periodic over the key frames.
All arrays are float32 vertices (V, 3) and uint32 triangle indices (N, 3).
"""
from __future__ import annotations

import functools
import math

import numpy as np

UP = (0.0, 0.0, 1.0)


def heightfield(n: int = 129, seed: int = 0, n_sines: int = 4, amp: float = 0.025):
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 1.0, n, dtype=np.float64)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    Z = np.zeros_like(X)
    for _ in range(n_sines):
        f = rng.uniform(1.0, 8.0)
        th = rng.uniform(0.0, 2.0 * math.pi)
        ph = rng.uniform(0.0, 2.0 * math.pi)
        Z += amp * np.sin(2.0 * math.pi * f * (math.cos(th) * X + math.sin(th) * Y) + ph)
    verts = np.stack([X, Y, Z], axis=-1).reshape(-1, 3).astype(np.float32)
    j, i = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    v00 = (j * n + i).reshape(-1)
    v10 = v00 + 1
    v01 = v00 + n
    v11 = v01 + 1
    tris = np.empty((v00.size * 2, 3), np.uint32)
    tris[0::2] = np.stack([v00, v10, v11], axis=1)
    tris[1::2] = np.stack([v00, v11, v01], axis=1)
    return verts, tris


@functools.lru_cache(maxsize=8)
def icosphere(level: int = 4):
    """Unit icosphere by midpoint subdivision: 20*4^level triangles, 10*4^level+2 vertices."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, np.float64), np.array(faces, np.uint32)


def clusters(n_tris: int, seed: int = 0, n_clusters: int = 64, sigma: float = 0.05,
             mu: float = math.log(0.01), s: float = 0.7, level: int = 4, ground: bool = True):
    rng = np.random.default_rng(seed)
    iv, iff = icosphere(level)
    tps = iff.shape[0]
    n_sphere = n_tris - (2 if ground else 0)
    if n_sphere < 0:
        raise ValueError("n_tris too small")
    full, rem = divmod(n_sphere, tps)
    nsph = full + (1 if rem else 0)
    means = rng.uniform(0.0, 1.0, (n_clusters, 3))
    which = rng.integers(0, n_clusters, nsph)
    centres = means[which] + rng.normal(0.0, sigma, (nsph, 3))
    radii = np.exp(rng.normal(mu, s, nsph))
    V = (centres[:, None, :] + radii[:, None, None] * iv[None, :, :]).reshape(-1, 3)
    F = (iff[None, :, :] + (np.arange(nsph, dtype=np.uint32) * iv.shape[0])[:, None, None]).reshape(-1, 3)
    F = F[:n_sphere]
    if ground:
        g0 = V.shape[0]
        gv = np.array([[-0.5, -0.5, 0.0], [1.5, -0.5, 0.0], [1.5, 1.5, 0.0], [-0.5, 1.5, 0.0]])
        V = np.concatenate([V, gv])
        F = np.concatenate([F, np.array([[g0, g0 + 1, g0 + 2], [g0, g0 + 2, g0 + 3]], np.uint32)])
    return V.astype(np.float32), np.ascontiguousarray(F, np.uint32)


def curl_keyframes(verts: np.ndarray, n_keyframes: int = 16, amp: float = 0.02, octaves: int = 4,
                   seed: int = 0, base_freq: float = 2.0):
    """Key frames k = 0..K-1: verts + amp * curl(psi)(p, k/K), psi a sum of `octaves`
    octaves of random plane waves (vector potential), periodic in k/K."""
    rng = np.random.default_rng(seed)
    P = verts.astype(np.float64)
    frames = np.empty((n_keyframes,) + verts.shape, np.float32)
    waves = []
    for o in range(octaves):
        f = base_freq * (2.0 ** o) * 2.0 * math.pi
        for comp in range(3):
            for _ in range(2):
                kdir = rng.normal(size=3)
                kdir /= np.linalg.norm(kdir)
                waves.append((comp, f * kdir, rng.uniform(0, 2 * math.pi), int(rng.integers(1, 3)), 0.5 ** o))
    for k in range(n_keyframes):
        tau = k / n_keyframes
        curl = np.zeros_like(P)
        for comp, kv, ph, om, a in waves:
            arg = P @ kv + ph + 2.0 * math.pi * om * tau
            g = a * np.cos(arg)[:, None] * kv[None, :]   # gradient of psi_comp
            # curl of (psi_x, psi_y, psi_z): contributions of one component
            if comp == 0:
                curl[:, 1] += g[:, 2]
                curl[:, 2] -= g[:, 1]
            elif comp == 1:
                curl[:, 0] -= g[:, 2]
                curl[:, 2] += g[:, 0]
            else:
                curl[:, 0] += g[:, 1]
                curl[:, 1] -= g[:, 0]
        if k == 0:
            scale = amp / max(1e-12, float(np.sqrt((curl ** 2).sum(1)).max()))
        frames[k] = (P + scale * curl).astype(np.float32)
    return frames


def camera_c1(res=(256, 256)):
    """Config-1 pinhole: (0.5,-0.8,0.9) looking at (0.5,0.5,0), 60 deg vertical FOV, +z up."""
    pos = np.array([0.5, -0.8, 0.9], np.float32)
    look = np.array([0.5, 0.5, 0.0], np.float32)
    return dict(position=pos, orientation=(look - pos), up=UP, fov=60.0, res_x=res[0], res_y=res[1])


def camera_at_bounds(verts: np.ndarray, res):
    """Config-1 camera position aimed at the centre of the scene bounds."""
    pos = np.array([0.5, -0.8, 0.9], np.float32)
    c = 0.5 * (verts.min(0) + verts.max(0))
    return dict(position=pos, orientation=(c - pos).astype(np.float32), up=UP, fov=60.0, res_x=res[0],
                res_y=res[1])


def config_scene(name: str, seed: int = 0):
    """Scenes of the benchmark configurations: 'c1' heightfield, 'c2' 1M clusters, 'c3' 2M clusters."""
    if name == "c1":
        return heightfield(129, seed)
    if name == "c2":
        return clusters(1_048_576, seed)
    if name == "c3":
        return clusters(2_097_152, seed)
    raise ValueError(name)


def heightfield_tris(n_tris: int, seed: int = 0):
    """Heightfield of the config-1 kind with exactly n_tris triangles: the smallest
    square grid holding them, its last triangles dropped."""
    n = max(2, int(math.ceil(math.sqrt(n_tris / 2.0))) + 1)
    v, f = heightfield(n, seed)
    return v, np.ascontiguousarray(f[:n_tris])


def batch_scenes(n_scenes: int = 256, seed: int = 0, tri_range=(1_000, 500_000), px_range=(64 * 64, 512 * 512)):
    """Batched-workload scenes: triangle counts log-uniform in tri_range, each a heightfield
    or a cluster scene (coin flip), a square image whose pixel count is log-uniform in
    px_range, camera as camera_at_bounds.  Returns dicts with v, f, cam."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        nt = int(round(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))))
        npx = math.exp(rng.uniform(math.log(px_range[0]), math.log(px_range[1])))
        side = max(8, int(round(math.sqrt(npx))))
        sseed = int(rng.integers(0, 2**31 - 1))
        if rng.random() < 0.5:
            v, f = heightfield_tris(nt, sseed)
            kind = "heightfield"
        else:
            v, f = clusters(max(nt, 3), sseed)
            kind = "clusters"
        out.append(dict(v=v, f=f, cam=camera_at_bounds(v, (side, side)), kind=kind))
    return out


def curl_keyframes_torch(verts: np.ndarray, n_keyframes: int = 16, amp: float = 0.02, octaves: int = 4,
                         seed: int = 0, base_freq: float = 2.0, device: str = "cuda"):
    """curl_keyframes evaluated with torch (float64) on `device`: the same waves and
    formula, for large meshes (the bench's data generation, not the engine)."""
    import torch
    rng = np.random.default_rng(seed)
    P = torch.from_numpy(verts.astype(np.float64)).to(device)
    waves = []
    for o in range(octaves):
        f = base_freq * (2.0 ** o) * 2.0 * math.pi
        for comp in range(3):
            for _ in range(2):
                kdir = rng.normal(size=3)
                kdir /= np.linalg.norm(kdir)
                waves.append((comp, f * kdir, rng.uniform(0, 2 * math.pi), int(rng.integers(1, 3)), 0.5 ** o))
    frames = np.empty((n_keyframes,) + verts.shape, np.float32)
    scale = None
    for k in range(n_keyframes):
        tau = k / n_keyframes
        curl = torch.zeros_like(P)
        for comp, kv, ph, om, a in waves:
            kt = torch.tensor(kv, dtype=torch.float64, device=device)
            arg = P @ kt + ph + 2.0 * math.pi * om * tau
            g = a * torch.cos(arg)[:, None] * kt[None, :]
            if comp == 0:
                curl[:, 1] += g[:, 2]
                curl[:, 2] -= g[:, 1]
            elif comp == 1:
                curl[:, 0] -= g[:, 2]
                curl[:, 2] += g[:, 0]
            else:
                curl[:, 0] += g[:, 1]
                curl[:, 1] -= g[:, 0]
        if scale is None:
            scale = amp / max(1e-12, float(torch.sqrt((curl ** 2).sum(1)).max()))
        frames[k] = (P + scale * curl).float().cpu().numpy()
    return frames


def served_scenes(n_scenes: int = 64, seed: int = 0, tri_range=(10_000, 4_000_000), n_keyframes: int = 16,
                  device: str | None = None):
    """Served-workload pool: cluster scenes as the key-frame configuration, triangle counts
    log-uniform in tri_range, n_keyframes curl-noise key frames each.  Returns
    (keyframes [K, V, 3] float32, faces [N, 3] uint32) pairs."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_scenes):
        nt = int(round(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))))
        sseed = int(rng.integers(0, 2**31 - 1))
        v, f = clusters(nt, sseed)
        if device:
            kf = curl_keyframes_torch(v, n_keyframes, amp=0.02, octaves=4, seed=sseed, device=device)
        else:
            kf = curl_keyframes(v, n_keyframes, amp=0.02, octaves=4, seed=sseed)
        out.append((kf, f))
    return out


INSTANCE_DTYPE = np.dtype([("obj", "<u4"), ("m", "<f4", 12), ("bmin", "<f4", 3), ("bmax", "<f4", 3)])


def instance_record(obj: int, to_world: np.ndarray, obj_lo, obj_hi):
    """An instance of an object: the world -> object rows of the reference's instances
    file (x' = m0 x + m1 y + m2 z + m3, ...) and the world box of the object's box corners.
    to_world: 3x4 object -> world map (float64)."""
    W = np.asarray(to_world, np.float64)
    A, T = W[:, :3], W[:, 3]
    Ai = np.linalg.inv(A)
    M = np.concatenate([Ai, (-Ai @ T)[:, None]], axis=1)
    lo, hi = np.asarray(obj_lo, np.float64), np.asarray(obj_hi, np.float64)
    corners = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    wc = corners @ A.T + T
    span = np.abs(wc).max() + 1.0
    rec = np.zeros((), INSTANCE_DTYPE)
    rec["obj"] = obj
    rec["m"] = M.reshape(-1).astype(np.float32)
    rec["bmin"] = (wc.min(0) - 1e-5 * span).astype(np.float32)   # outward: the box holds the object
    rec["bmax"] = (wc.max(0) + 1e-5 * span).astype(np.float32)
    return rec


def instanced_scene(n_objects: int = 16, n_instances: int = 1024, seed: int = 0, tri_range=(320, 20_480),
                    world: float = 1.0, scale_range=(0.02, 0.08)):
    """Seeded instanced scene: objects (icospheres of levels 2-5 and heightfield tiles, each
    centred at its origin with extent about 1) and instances with random rotations,
    uniform scales and positions in [0, world]^3 (ground objects lie flat).  Returns
    (vertices, faces, object triangle counts, instance records)."""
    rng = np.random.default_rng(seed)
    verts, faces, counts, boxes = [], [], [], []
    nv = 0
    for k in range(n_objects):
        target = int(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1]))))
        if k % 2 == 0:
            level = max(2, min(5, int(round(math.log(max(target, 80) / 20.0, 4)))))
            v, f = icosphere(level)
            v = np.asarray(v, np.float64) * 0.5
        else:
            n = max(3, int(math.sqrt(target / 2.0)) + 1)
            v, f = heightfield(n, int(rng.integers(1 << 30)), amp=0.05)
            v = np.asarray(v, np.float64) - np.array([0.5, 0.5, 0.0])
        v = v.astype(np.float32)
        verts.append(v)
        faces.append(np.asarray(f, np.uint32) + nv)
        counts.append(len(f))
        boxes.append((v.min(0), v.max(0)))
        nv += v.shape[0]
    inst = np.zeros(n_instances, INSTANCE_DTYPE)
    for i in range(n_instances):
        obj = int(rng.integers(0, n_objects))
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, c, d = q
        R = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                      [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                      [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])
        s = math.exp(rng.uniform(math.log(scale_range[0]), math.log(scale_range[1])))
        T = rng.uniform(0.0, world, 3)
        inst[i] = instance_record(obj, np.concatenate([R * s, T[:, None]], axis=1), *boxes[obj])
    return np.concatenate(verts), np.concatenate(faces), np.asarray(counts, np.uint32), inst
