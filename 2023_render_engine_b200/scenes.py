"""Seeded synthetic scenes and ray sets (the reference ships no benchmark scenes).

* cornell_box(): closed box [-1,1]^3 of 5 quads (10 triangles), a 0.5x0.5 ceiling light
  at y = 0.99 (2 triangles), a Lambertian and a glass sphere of radius 0.3.
* stress_scene(): icosphere subdivided 8 times (1,310,720 triangles) with 3-octave value
  noise radial displacement of amplitude 0.05, inside the Cornell box.
* random_rays(): origins uniform in [-1,1]^3, directions uniform on the sphere.

Everything is float32 and reproducible from the seed on any machine with this numpy.
"""
from __future__ import annotations

import math

import numpy as np

# material slots used by the generators (indices into the material table)
MAT_WHITE, MAT_RED, MAT_GREEN, MAT_LIGHT, MAT_DIFFUSE_SPHERE, MAT_GLASS, MAT_GGX = range(7)


def quad(p0, p1, p2, p3):
    v = np.array([p0, p1, p2, p3], dtype=np.float32)
    return v, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)


def cornell_walls():
    """The five walls of the box [-1,1]^3 (open towards +z) and the ceiling light quad."""
    walls = {
        "floor": (quad((-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1)), MAT_WHITE),
        "ceiling": (quad((-1, 1, 1), (-1, 1, -1), (1, 1, -1), (1, 1, 1)), MAT_WHITE),
        "back": (quad((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)), MAT_WHITE),
        "left": (quad((-1, -1, 1), (-1, -1, -1), (-1, 1, -1), (-1, 1, 1)), MAT_RED),
        "right": (quad((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)), MAT_GREEN),
        "light": (quad((-0.25, 0.99, 0.25), (-0.25, 0.99, -0.25), (0.25, 0.99, -0.25), (0.25, 0.99, 0.25)),
                  MAT_LIGHT),
    }
    return walls


def sphere_matrices(center, radius):
    """objectToWorld = translate(center) * rotateZ(90) as Sphere(Point3f,Float) builds it
    (shapes/Sphere.cu:233-245), and its inverse (rigid: R^T, -R^T t)."""
    ang = np.float32(np.float64(np.float32(90.0) * np.float32(math.pi)) / 180.0)
    s, c = np.float32(math.sin(ang)), np.float32(math.cos(ang))
    r = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], dtype=np.float32)
    t = np.asarray(center, dtype=np.float32)
    o2w = np.eye(4, dtype=np.float32)
    o2w[:3, :3] = r
    o2w[:3, 3] = t
    w2o = np.eye(4, dtype=np.float32)
    w2o[:3, :3] = r.T
    w2o[:3, 3] = -(r.T @ t)
    return o2w, w2o


def cornell_box():
    """Config 0 geometry: meshes (list of (vertices, indices, material)) and spheres."""
    meshes = [(v, i, m) for (v, i), m in cornell_walls().values()]
    spheres = [
        {"center": (-0.4, -0.7, -0.3), "radius": 0.3, "material": MAT_DIFFUSE_SPHERE, "glass": False},
        {"center": (0.4, -0.7, 0.3), "radius": 0.3, "material": MAT_GLASS, "glass": True},
    ]
    return {"meshes": meshes, "spheres": spheres}


def icosphere(subdiv: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
        key = lo * nv + hi
        uk, inv = np.unique(key, return_inverse=True)
        mid = (v[uk // nv] + v[uk % nv]) * 0.5
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = (inv + nv).reshape(3, -1).T  # midpoints of edges 01, 12, 20
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1), np.stack([ca, bc, c], 1),
                            np.stack([ab, bc, ca], 1)])
        v = np.concatenate([v, mid])
    return v, f


def value_noise(p: np.ndarray, seed: int, octaves=3, base_freq=4.0) -> np.ndarray:
    """Seeded lattice value noise in [-1,1] (smoothstep trilinear), octave sum normalised."""
    rng = np.random.default_rng(seed)
    out = np.zeros(p.shape[0])
    norm = 0.0
    for o in range(octaves):
        freq = base_freq * (2 ** o)
        amp = 0.5 ** o
        g = int(math.ceil(2 * freq)) + 3
        lat = rng.uniform(-1.0, 1.0, size=(g, g, g))
        q = (p + 1.0) * freq  # p in [-1,1] -> [0, 2 freq]
        i0 = np.floor(q).astype(np.int64)
        fr = q - i0
        w = fr * fr * (3 - 2 * fr)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    val = lat[i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz]
                    wt = (w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1]) * \
                         (w[:, 2] if dz else 1 - w[:, 2])
                    acc += wt * val
        out += amp * acc
        norm += amp
    return out / norm


def displaced_icosphere(subdiv=8, radius=0.55, amplitude=0.05, seed=1):
    v, f = icosphere(subdiv)
    n = value_noise(v, seed)
    v = v * (radius * (1.0 + amplitude * n))[:, None]
    return v.astype(np.float32), f.astype(np.uint32)


def ggx_block_roughness(ntri: int, seed=2, block=64):
    """Roughness uniform in [0.05, 0.5] per block of 64 consecutive triangles."""
    rng = np.random.default_rng(seed)
    nb = (ntri + block - 1) // block
    return np.repeat(rng.uniform(0.05, 0.5, nb).astype(np.float32), block)[:ntri]


def stress_scene(subdiv=8, seed=1):
    """Config 1 geometry: the displaced icosphere (GGX) inside the Cornell box walls + light."""
    v, f = displaced_icosphere(subdiv=subdiv, seed=seed)
    meshes = [(wv, wi, m) for (wv, wi), m in cornell_walls().values()]
    meshes.append((v, f, MAT_GGX))
    return {"meshes": meshes, "spheres": [], "roughness": ggx_block_roughness(f.shape[0])}


def random_rays(n: int, seed=7, lo=-1.0, hi=1.0):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    z = rng.uniform(-1.0, 1.0, size=n)
    phi = rng.uniform(0.0, 2 * math.pi, size=n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([s * np.cos(phi), s * np.sin(phi), z], 1).astype(np.float32)
    return o, d


def flatten(scene):
    """Concatenates meshes into one triangle soup in scene order (global triangle ids)."""
    vs, fs, mats = [], [], []
    base = 0
    for v, f, m in scene["meshes"]:
        vs.append(v)
        fs.append(f.astype(np.uint32) + base)
        mats.append(np.full(f.shape[0], m, np.uint32))
        base += v.shape[0]
    return np.concatenate(vs), np.concatenate(fs), np.concatenate(mats)


def subdivided_box(lo, hi, n):
    """Axis-aligned box [lo, hi] with each face split into an n x n grid (12 n^2 triangles),
    outward-facing winding."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    vs, fs = [], []
    g = np.linspace(0.0, 1.0, n + 1)
    U, V = np.meshgrid(g, g, indexing="ij")
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel(), idx[:-1, 1:].ravel()
    quad = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    base = 0
    for axis in range(3):
        u_ax, v_ax = (axis + 1) % 3, (axis + 2) % 3
        for side, val in ((0, lo[axis]), (1, hi[axis])):
            P = np.zeros((U.size, 3))
            P[:, axis] = val
            P[:, u_ax] = lo[u_ax] + U.ravel() * (hi[u_ax] - lo[u_ax])
            P[:, v_ax] = lo[v_ax] + V.ravel() * (hi[v_ax] - lo[v_ax])
            f = quad if side == 1 else quad[:, ::-1]
            vs.append(P)
            fs.append(f + base)
            base += P.shape[0]
    return np.concatenate(vs).astype(np.float32), np.concatenate(fs).astype(np.uint32)


def guiding_room(seed=3, target_triangles=200_000):
    """Config 2 geometry: a closed room [-2,2]x[0,2.5]x[-2,2] split by a wall at z = 1 with a
    0.2-wide vertical gap; a 0.3x0.3 emitter (Le = 20) behind the wall; seeded random boxes
    (each 12 n^2 triangles with n chosen so a box has 20..2000 triangles, sizes log-uniform in
    [0.05, 1]) on the floor until about `target_triangles` triangles. Per-box material:
    Lambertian albedo U[0.2, 0.9], or (30%) GGX roughness U[0.1, 0.4].
    Returns meshes [(v, f, material_key)] and a material list (dicts for configs.py)."""
    rng = np.random.default_rng(seed)
    meshes, mats = [], []

    def add(v, f, m):
        mats.append(m)
        meshes.append((v, f, len(mats) - 1))

    wall = dict(kind="lambert", albedo=(0.7, 0.7, 0.7))
    room = subdivided_box((-2, 0, -2), (2, 2.5, 2), 2)
    add(room[0], room[1][:, ::-1].copy(), wall)  # inward-facing
    # dividing wall at z = 1 (0.1 thick) with a gap 0.2 wide at x in [0.4, 0.6]
    add(*subdivided_box((-2, 0, 0.95), (0.4, 2.5, 1.05), 2), wall)
    add(*subdivided_box((0.6, 0, 0.95), (2, 2.5, 1.05), 2), wall)
    # the emitter behind the wall, facing -z towards the wall
    lv = np.array([[0.35, 1.0, 1.8], [0.65, 1.0, 1.8], [0.65, 1.3, 1.8], [0.35, 1.3, 1.8]], np.float32)
    add(lv, np.array([[0, 2, 1], [0, 3, 2]], np.uint32), dict(kind="light", emission=(20.0, 20.0, 20.0)))
    ntri = sum(f.shape[0] for _, f, _ in meshes)
    while ntri < target_triangles:
        size = np.exp(rng.uniform(np.log(0.05), np.log(1.0), 3))
        x, z = rng.uniform(-1.9, 1.9 - size[0]), rng.uniform(-1.9, 0.9 - size[2])
        lo = np.array([x, 0.0, z])
        hi = lo + size
        n = int(rng.integers(1, 13))  # 12 n^2 in [12 .. 1728]
        n = max(n, 2)                 # at least 48 triangles
        v, f = subdivided_box(lo, hi, n)
        if rng.uniform() < 0.3:
            m = dict(kind="ggx", roughness=float(rng.uniform(0.1, 0.4)))
        else:
            m = dict(kind="lambert", albedo=tuple(float(a) for a in rng.uniform(0.2, 0.9, 3)))
        add(v, f, m)
        ntri += f.shape[0]
    return meshes, mats


def terrain_grid(n=1000, half=4.0, amplitude=0.35, seed=11, octaves=5, base_freq=1.5):
    """Height-field terrain over [-half, half]^2 in xz: an (n+1)^2 vertex grid, 2 n^2
    triangles facing +y, heights amplitude * value noise of (x, z) / half. Returns (v, f, height)
    with height(x, z) the same field at arbitrary points."""
    g = np.linspace(-half, half, n + 1)
    X, Z = np.meshgrid(g, g, indexing="ij")

    def height(x, z):
        x = np.asarray(x, np.float64).ravel()
        z = np.asarray(z, np.float64).ravel()
        p = np.stack([x / half, z / half, np.zeros_like(x)], 1)
        return amplitude * value_noise(p, seed, octaves=octaves, base_freq=base_freq)

    Y = height(X, Z).reshape(X.shape)
    v = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel(), idx[:-1, 1:].ravel()
    # (x, z) grid with x along the first index: (a, d, c) and (a, c, b) wind counter-clockwise
    # seen from +y
    f = np.concatenate([np.stack([a, d, c], 1), np.stack([a, c, b], 1)])
    return v.astype(np.float32), f.astype(np.uint32), height


def photon_terrain(seed=11, n=1000):
    """Config 4 geometry: the displaced terrain (2 n^2 triangles; 2M at n = 1000), 16 glass
    spheres of radius U[0.1, 0.4] resting on it without overlapping, and a 1.2 x 0.3 x 0.8
    subsurface slab sunk 0.05 into it near the centre. Returns terrain (v, f), slab (v, f) and
    the spheres [(centre, radius)]."""
    rng = np.random.default_rng(seed + 1)
    tv, tf, height = terrain_grid(n=n, seed=seed)
    spheres = []
    while len(spheres) < 16:
        r = float(rng.uniform(0.1, 0.4))
        x, z = rng.uniform(-2.5, 2.5, 2)
        if abs(x) < 1.0 and abs(z) < 0.8:
            continue  # keep the slab's footprint clear
        if any((x - c[0]) ** 2 + (z - c[2]) ** 2 < (r + rr + 0.05) ** 2 for c, rr in spheres):
            continue
        y = float(height([x], [z])[0]) + r + 0.02
        spheres.append(((float(x), y, float(z)), r))
    h0 = float(height([0.0], [0.2])[0]) - 0.05
    sv, sf = subdivided_box((-0.6, h0, -0.2), (0.6, h0 + 0.3, 0.6), 1)
    return (tv, tf), (sv, sf), spheres
