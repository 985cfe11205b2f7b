"""Pins the C restatement (oracle/rt_oracle.c) to the reference renderer's own code:
against the golden fixtures generated by the reference build, and against the live
reference harness when it is available. CPU only."""
import importlib

import numpy as np
import pytest

import cases
from conftest import GOLDEN

S = importlib.import_module("2023_render_engine_b200.scenes")


def _golden(name):
    z = np.load(GOLDEN / name)
    return z


def _unpack(z, key):
    return {k.split("__", 1)[1]: z[k] for k in z.files if k.startswith(key + "__")}


@pytest.mark.parametrize("key", ["soup1000", "soup20000", "grids"])
def test_restated_tree_matches_golden(restated, key):
    g = _unpack(_golden("trace_small.npz"), key)
    b = restated.bvh(g["v"], g["f"])
    ex = b.export()
    assert np.array_equal(ex["codes"], g["codes"])
    assert np.array_equal(ex["sorted"], g["sorted"])


@pytest.mark.parametrize("key", ["soup1000", "soup20000", "grids"])
def test_restated_trace_matches_golden(restated, key):
    g = _unpack(_golden("trace_small.npz"), key)
    b = restated.bvh(g["v"], g["f"])
    ids, t = b.intersect(g["o"], g["d"])
    assert np.array_equal(ids, g["ids"])
    hit = ids >= 0
    assert np.array_equal(t[hit], g["t"][hit])


def test_restated_spheres_match_golden(restated):
    g = _golden("spheres_cornell.npz")
    n = g["o"].shape[0]
    for shadow, ids_key, t_key in [(False, "ids", "t"), (True, "ids_shadow", "t_shadow")]:
        ids = np.full(n, -1, np.int32)
        ts = np.full(n, np.inf, np.float32)
        for i in range(len(g["radii"])):
            if shadow and i == 1:  # the glass sphere is transparent to shadow rays
                continue
            for r in range(n):
                hit, t = restated.sphere_intersects(g[f"w2o{i}"], g["radii"][i], g["o"][r], g["d"][r],
                                                    hit_offset=ts[r])
                if hit:
                    ids[r], ts[r] = i, t
        assert np.array_equal(ids, g[ids_key])
        assert np.array_equal(ts[ids >= 0], g[t_key][ids >= 0])


def test_restated_knn_matches_golden(restated):
    g = _golden("knn_small.npz")
    k = int(g["k"])
    idx, dist, cnt = restated.knn(g["pos"], g["shape"], g["q"], g["qshape"], k, float(g["radius"]))
    assert np.array_equal(cnt, g["count"])
    for i in range(len(cnt)):
        assert set(idx[i, :cnt[i]].tolist()) == set(g["idx"][i, :cnt[i]].tolist())


def test_tie_rank_is_reference_visit_order(restated, refo):
    """The restated static rank reproduces the order in which the reference traversal
    tests triangles: a ray that hits every box sees them in rank order."""
    v, f = cases.soup(257, 5)
    b = restated.bvh(v, f)
    r = b.tie_rank()
    assert sorted(r.tolist()) == list(range(257))
    ex = refo.bvh(v, f).export()
    n = 257
    # recompute the visit order from the exported reference tree (left/right arrays)
    order = []
    stack = [int(ex["root"])]
    while stack:
        node = stack.pop()
        for c in (int(ex["left"][node]), int(ex["right"][node])):
            if ex["objectIds"][c] >= 0:
                order.append(int(ex["objectIds"][c]))
            else:
                stack.append(c)
    assert [int(x) for x in np.argsort(r)] == order
    assert n == len(order)


@pytest.mark.parametrize("nt,seed", [(2, 1), (3, 2), (17, 3), (513, 4), (5000, 5)])
def test_restated_vs_live_reference(restated, refo, nt, seed):
    v, f = cases.soup(nt, seed, size=0.2)
    rb, ob = refo.bvh(v, f), restated.bvh(v, f)
    er, eo = rb.export(), ob.export()
    assert np.array_equal(er["codes"], eo["codes"])
    assert np.array_equal(er["sorted"], eo["sorted"])
    assert np.array_equal(er["boxes"], eo["boxes"])
    o, d = S.random_rays(3000, seed=seed + 100, lo=-1.3, hi=1.3)
    for shadow in (False, True):
        a = rb.intersect(o, d, shadow=shadow)
        b, _ = ob.intersect(o, d, shadow=shadow)
        assert np.array_equal(a, b)


def test_restated_edge_cases_vs_live_reference(restated, refo):
    v, f = cases.stacked_grids()
    tr = np.zeros(f.shape[0], np.uint8)
    tr[-2:] = 1  # the tilted quad is transparent to shadow rays
    rb, ob = refo.bvh(v, f, tr), restated.bvh(v, f, tr)
    o, d = cases.edge_rays(9)
    for shadow in (False, True):
        a = rb.intersect(o, d, shadow=shadow)
        b, _ = ob.intersect(o, d, shadow=shadow)
        assert np.array_equal(a, b)
    # finite tmax
    tm = np.random.default_rng(2).uniform(0.1, 3.0, o.shape[0]).astype(np.float32)
    assert np.array_equal(rb.intersect(o, d, tmax=tm), ob.intersect(o, d, tmax=tm)[0])


def test_restated_triangle_offset_quirk(restated, refo):
    """Triangle::intersects lowers the running offset before its error-bound rejection."""
    v = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0], [-1, -1, 1], [1, -1, 1], [0, 1, 1]], np.float32)
    f = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    rb, ob = refo.bvh(v, f), restated.bvh(v, f)
    for z0 in [-1e-9, -1e-8, -1e-7, -1e-6, -1e-3]:
        o = np.array([0.1, 0.0, z0], np.float32)
        d = np.array([0.0, 0.0, 1.0], np.float32)
        assert rb.triangle_intersects(0, o, d) == ob.triangle_intersects(0, o, d)
        assert rb.triangle_intersects(1, o, d, hit_offset=2e-9) == ob.triangle_intersects(1, o, d, hit_offset=2e-9)


def test_restated_spheres_vs_live_reference(restated, refo):
    from oracle import bindings

    rng = np.random.default_rng(4)
    centers = rng.uniform(-1, 1, (6, 3)).astype(np.float32)
    radii = rng.uniform(0.05, 0.5, 6).astype(np.float32)
    rs = bindings.RefSpheres(refo, centers, radii, np.zeros(6, np.uint8))
    o, d = S.random_rays(2000, seed=8, lo=-1.5, hi=1.5)
    ids, t = rs.intersect(o, d)
    for r in range(0, 2000, 7):
        best, bi = np.inf, -1
        for i in range(6):
            hit, tt = restated.sphere_intersects(rs.matrices(i)[1], radii[i], o[r], d[r], hit_offset=best)
            if hit:
                best, bi = tt, i
        assert bi == ids[r]
        if bi >= 0:
            assert best == t[r]


def test_restated_knn_vs_live_reference(restated, refo):
    from oracle import bindings

    rng = np.random.default_rng(5)
    pos = rng.normal(0, 0.5, (30000, 3)).astype(np.float32)
    shp = rng.integers(0, 3, 30000).astype(np.int32)
    q = rng.normal(0, 0.5, (300, 3)).astype(np.float32)
    for k, radius, qs in [(1, 10.0, None), (50, 0.2, rng.integers(-1, 3, 300).astype(np.int32)), (100, 100.0, None)]:
        kd = bindings.RefKdTree(refo, pos, shp)
        a, ca = kd.knn(q, k, radius, qs)
        b, _, cb = restated.knn(pos, shp, q, qs, k, radius)
        assert np.array_equal(ca, cb)
        for i in range(300):
            assert set(a[i, :ca[i]].tolist()) == set(b[i, :cb[i]].tolist())
