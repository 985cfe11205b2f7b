"""Seeded closest-hit cases shared by the golden-fixture generator and the tests."""
from __future__ import annotations

import importlib

import numpy as np

S = importlib.import_module("2023_render_engine_b200.scenes")


def soup(nt: int, seed: int, spread=1.0, size=0.1):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (nt, 3)).astype(np.float32)
    v = (c[:, None, :] + rng.normal(0, size, (nt, 3, 3))).astype(np.float32).reshape(-1, 3)
    return v, np.arange(nt * 3, dtype=np.uint32).reshape(-1, 3)


def grid_mesh(n=8, z=0.0):
    """Regular grid of 2n^2 triangles on [-1,1]^2 at height z, vertices on multiples of 2/n
    (exactly representable), so rays through grid lines produce exact edge ties."""
    xs = np.linspace(-1, 1, n + 1, dtype=np.float32)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    v = np.stack([X.ravel(), Y.ravel(), np.full(X.size, z, np.float32)], 1).astype(np.float32)
    f = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = i * (n + 1) + j, (i + 1) * (n + 1) + j, (i + 1) * (n + 1) + j + 1, i * (n + 1) + j + 1
            f.append([a, b, c])
            f.append([a, c, d])
    return v, np.array(f, np.uint32)


def stacked_grids():
    """Two parallel grids (z = 0 and z = 0.5) plus a tilted quad: ties, coplanar layers."""
    v0, f0 = grid_mesh(8, 0.0)
    v1, f1 = grid_mesh(4, 0.5)
    v2 = np.array([[-0.6, -0.6, -0.4], [0.6, -0.6, 0.2], [0.6, 0.6, 0.2], [-0.6, 0.6, -0.4]], np.float32)
    f2 = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    v = np.concatenate([v0, v1, v2])
    f = np.concatenate([f0, f1 + len(v0), f2 + len(v0) + len(v1)])
    return v, f


def edge_rays(seed=3):
    """Rays aimed at grid lines and vertices (exact ties), axis-aligned rays (zero direction
    components), rays starting a hair below a surface (offset smaller than the error bound),
    and random rays."""
    rng = np.random.default_rng(seed)
    o, d = [], []
    g = np.linspace(-1, 1, 9, dtype=np.float32)
    for x in g:
        for y in g:
            o.append([x, y, 2.0]); d.append([0, 0, -1])          # straight down through vertices
            o.append([x, y + 0.125, 2.0]); d.append([0, 0, -1])  # through edge midpoints
            o.append([x, y, -2.0]); d.append([0, 0, 1])
    for _ in range(300):
        x, y = rng.choice(g), rng.uniform(-1, 1)
        o.append([x, y, 1.5]); d.append([0.0, rng.uniform(-0.3, 0.3), -1])  # in the plane x = grid line
    for _ in range(300):  # just below the z=0 grid, going up: near-zero offsets
        x, y = rng.uniform(-0.9, 0.9, 2)
        o.append([x, y, -float(rng.choice([1e-9, 1e-8, 1e-7, 0.0]))]); d.append(list(rng.uniform(-0.5, 0.5, 2)) + [1.0])
    for _ in range(300):  # axis-aligned in x or y
        ax = rng.integers(0, 2)
        dd = [0.0, 0.0, 0.0]
        dd[ax] = float(rng.choice([-1.0, 1.0]))
        o.append(list(rng.uniform(-1.2, 1.2, 2)) + [float(rng.choice([0.0, 0.5, 0.25, 0.1]))]); d.append(dd)
    ro, rd = S.random_rays(2000, seed=seed + 1, lo=-1.5, hi=1.5)
    o = np.concatenate([np.array(o, np.float32), ro])
    d = np.concatenate([np.array(d, np.float32), rd])
    return o.astype(np.float32), d.astype(np.float32)


def cornell_soup():
    sc = S.cornell_box()
    v, f, m = S.flatten(sc)
    return v, f, m, sc["spheres"]
