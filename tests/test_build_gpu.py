"""The device build of the acceleration structures (RT_BUILD_DEVICE, the default) against the
host build (RT_BUILD_HOST): the same bytes for the 8-wide nodes, the triangle records (with
the reference traversal ranks) and the reference tree's boxes, on edge sizes, random soups,
duplicated triangles, the Cornell box and the 1.31M-triangle BVH-stress mesh; and the same
closest hits. The host build is the restatement the device build is checked against; the
reference-order tree it holds is pinned to the reference by the trace parity tests."""
import importlib
import time

import numpy as np
import pytest

S = importlib.import_module("2023_render_engine_b200.scenes")
N = importlib.import_module("2023_render_engine_b200._native")

pytestmark = pytest.mark.gpu


def commit_both(core, ctx, meshes, transparent=()):
    out = []
    for mode in (N.RT_BUILD_HOST, N.RT_BUILD_DEVICE):
        sc = core.Scene(ctx)
        for i, (v, f) in enumerate(meshes):
            sc.add_mesh(v, f, shape_id=i, transparent=i in transparent)
        sc.set_build(mode)
        t0 = time.perf_counter()
        sc.commit()
        out.append((sc, time.perf_counter() - t0))
    return out


def assert_same_structures(a, b):
    na, ra, ba = a.export_bvh()
    nb, rb, bb = b.export_bvh()
    assert na.shape == nb.shape and ra.shape == rb.shape and ba.shape == bb.shape
    assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32)), "triangle records differ"
    assert np.array_equal(ba.view(np.uint32), bb.view(np.uint32)), "reference tree boxes differ"
    diff = np.nonzero((na != nb).any(1))[0]
    assert diff.size == 0, f"{diff.size} of {na.shape[0]} nodes differ, first {diff[:5]}"


def soup(rng, n, spread=1.0, size=0.05):
    c = rng.uniform(-spread, spread, (n, 1, 3))
    v = (c + rng.normal(0, size, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    return v, np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 9, 33, 1000, 65537])
def test_device_build_equals_host_build_on_soups(core, gpu_ctx, n):
    rng = np.random.default_rng(n)
    (h, _), (d, _) = commit_both(core, gpu_ctx, [soup(rng, n)])
    assert_same_structures(h, d)
    nodes, recs, _ = d.export_bvh()
    ids = np.sort(recs[:, 7].view(np.uint32))
    assert np.array_equal(ids, np.arange(n, dtype=np.uint32))  # every triangle in exactly one leaf
    assert np.array_equal(np.sort(recs[:, 3].view(np.uint32)), np.arange(n, dtype=np.uint32))  # ranks: a permutation


def test_device_build_with_duplicates_and_flat_geometry(core, gpu_ctx):
    """Coincident triangles (equal Morton codes and boxes), an axis-aligned flat grid (zero
    extents, tied areas) and transparent triangles."""
    rng = np.random.default_rng(5)
    v, f = soup(rng, 300)
    dup = (np.concatenate([v, v, v]), np.concatenate([f, f + len(v), f + 2 * len(v)]))
    g = np.linspace(-1, 1, 41)
    X, Y = np.meshgrid(g, g, indexing="ij")
    gv = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1).astype(np.float32)
    idx = np.arange(X.size).reshape(41, 41)
    a, b, c, d_ = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel(), idx[:-1, 1:].ravel()
    gf = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d_], 1)]).astype(np.uint32)
    (h, _), (d, _) = commit_both(core, gpu_ctx, [dup, (gv, gf)], transparent=(1,))
    assert_same_structures(h, d)


def test_device_build_cornell_and_trace(core, gpu_ctx):
    import torch

    sc_data = S.cornell_box()
    v, f, _ = S.flatten(sc_data)
    (h, _), (d, _) = commit_both(core, gpu_ctx, [(v, f)])
    assert_same_structures(h, d)
    o, dd = S.random_rays(1 << 16, seed=3)
    rays = core.make_rays(o, dd)
    hh = h.trace_closest_host(rays)
    hd = d.trace_closest_host(rays)
    assert np.array_equal(hh.view(np.uint32), hd.view(np.uint32))


def test_device_build_stress_mesh_is_identical_and_faster(core, gpu_ctx):
    v, f, _ = S.flatten(S.stress_scene())
    (h, th), (d, td) = commit_both(core, gpu_ctx, [(v, f)])
    assert_same_structures(h, d)
    hs, ds = h.stats(), d.stats()
    assert hs["bvh8_nodes"] == ds["bvh8_nodes"]
    # the device build replaces ~1 s of host threads; a second commit has warm kernels
    sc = core.Scene(gpu_ctx)
    sc.add_mesh(v, f)
    sc.commit()
    assert sc.stats()["build_ms"] < 0.5 * hs["build_ms"], (sc.stats()["build_ms"], hs["build_ms"])
