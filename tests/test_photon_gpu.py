"""Photon map k-nearest gathering and photon tracing through the C ABI, against the
reference's own kd-tree (nn::KDTree, compiled from its sources) and the C restatement."""
import importlib

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
S = importlib.import_module("2023_render_engine_b200.scenes")


def _sets(idx, cnt):
    return [set(idx[i, :cnt[i]].tolist()) for i in range(len(cnt))]


def test_knn_matches_golden(core, gpu_ctx):
    import torch

    g = np.load(GOLDEN / "knn_small.npz")
    pos = torch.from_numpy(g["pos"]).cuda()
    shp = torch.from_numpy(g["shape"]).cuda()
    m = core.PhotonMap.from_points(gpu_ctx, pos, shp).build()
    idx, dist, cnt = m.knn(torch.from_numpy(g["q"]).cuda(), int(g["k"]), float(g["radius"]),
                           torch.from_numpy(g["qshape"]).cuda())
    idx, cnt = idx.cpu().numpy(), cnt.cpu().numpy()
    assert np.array_equal(cnt, g["count"].astype(np.int32))
    assert _sets(idx, cnt) == _sets(g["idx"], g["count"])
    d = dist.cpu().numpy()
    for i in range(len(cnt)):
        assert np.all(np.diff(d[i, :cnt[i]]) >= 0)  # ascending


@pytest.mark.parametrize("n,k,radius,with_shape", [(1, 1, 10.0, False), (7, 50, 10.0, False),
                                                    (100000, 1, 100.0, False), (100000, 50, 0.1, True),
                                                    (300000, 100, 100.0, True), (50000, 128, 0.3, True)])
def test_knn_matches_reference_kdtree(core, gpu_ctx, refo, restated, n, k, radius, with_shape):
    import torch
    from oracle import bindings

    rng = np.random.default_rng(n + k)
    pos = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    pos[: n // 10] = np.round(pos[: n // 10], 2)  # a slab of duplicated coordinates
    shp = rng.integers(0, 3, n).astype(np.int32)
    q = rng.normal(0, 0.5, (2000, 3)).astype(np.float32)
    qs = rng.integers(-1, 3, 2000).astype(np.int32) if with_shape else None
    m = core.PhotonMap.from_points(gpu_ctx, torch.from_numpy(pos).cuda(), torch.from_numpy(shp).cuda()).build()
    gi, gd, gc = m.knn(torch.from_numpy(q).cuda(), k, radius, None if qs is None else torch.from_numpy(qs).cuda())
    gi, gd, gc = gi.cpu().numpy(), gd.cpu().numpy(), gc.cpu().numpy()
    kd = bindings.RefKdTree(refo, pos, shp)
    ri, rc = kd.knn(q, k, radius, qs)
    assert np.array_equal(gc, rc.astype(np.int32))
    # the sorted distances equal the brute-force restatement's; the sets equal the
    # reference's except for members tied at the k-th distance
    bi, bd, bc = restated.knn(pos, shp, q, qs, k, radius)
    for i in range(len(q)):
        assert np.array_equal(gd[i, :gc[i]], bd[i, :bc[i]])
        a, b = set(gi[i, :gc[i]].tolist()), set(ri[i, :rc[i]].tolist())
        if a != b:
            kth = bd[i, bc[i] - 1]
            dd = np.sqrt(((pos[list(a ^ b)] - q[i]) ** 2).sum(1))
            assert np.allclose(dd, kth, rtol=1e-6, atol=0)


def test_photon_trace_and_gather_on_cornell(core, gpu_ctx):
    import torch

    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, 32, 32)
    sc.add_point_light((0.0, 0.9, 0.0), (1.0, 1.0, 1.0), 5.0)
    sc.commit()
    pm, st = sc.trace_photons(200000, max_depth=30, seed=1)
    ph = pm.photons()
    assert st["emitted"] == 200000 and st["stored"] == len(ph) > 200000 * 0.5
    keys = ph["path"].astype(np.uint64) << 8 | ph["depth"]
    assert np.all(np.diff(keys.astype(np.int64)) > 0)  # (path, depth) order, no duplicates
    assert np.isfinite(ph["power"]).all() and (ph["power"] >= 0).all()
    # first-bounce photons of one light carry I * 4 pi / n (one light: p_l = 1)
    first = ph[ph["depth"] == 0]
    assert np.allclose(first["power"], 5.0 * 4 * np.pi / 200000, rtol=1e-5)
    # photons lie on the scene's surfaces: inside the box
    assert (np.abs(ph["pos"]) <= 1.0001).all()
    pm2, _ = sc.trace_photons(200000, max_depth=30, seed=1)
    assert np.array_equal(pm2.photons(), ph)  # deterministic
    pm.build()
    q = torch.from_numpy(ph["pos"][:1000].copy()).cuda()
    idx, dist, cnt = pm.knn(q, 50, 100.0)
    assert (cnt.cpu().numpy() == 50).all()
    assert (idx.cpu().numpy()[:, 0] >= 0).all()


def test_photon_trace_matches_cpu_restatement(core, gpu_ctx, restated):
    """Same per-photon PCG streams on both sides: the stored photons agree photon by photon
    up to float rounding (a few paths diverge where rounding flips a decision)."""
    from oracle import bindings

    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, 16, 16)
    lights = [((0.0, 0.9, 0.0), (1.0, 0.9, 0.8), 5.0), ((0.5, 0.5, 0.5), (0.2, 0.3, 1.0), 3.0)]
    for lp, c, i in lights:
        sc.add_point_light(lp, c, i)
    sc.commit()
    n = 20000
    pm, st = sc.trace_photons(n, max_depth=30, seed=9, flags=N.RT_RENDER_COMPAT)
    gpu = pm.photons()
    sc_data = S.cornell_box()
    v, f, m = S.flatten(sc_data)
    tri_shape = np.concatenate([np.full(fi.shape[0], i, np.int32) for i, (_, fi, _) in enumerate(sc_data["meshes"])])
    spheres = []
    for s in sc_data["spheres"]:
        o2w, w2o = S.sphere_matrices(s["center"], s["radius"])
        spheres.append({"o2w": o2w, "w2o": w2o, "radius": s["radius"], "material": s["material"]})
    orc = bindings.PathTracerOracle(restated, v, f, m, spheres, cfg.cornell_materials())
    cpu = orc.trace_photons(tri_shape, [100, 101], lights, n, max_depth=30, seed=9, flags=N.RT_RENDER_COMPAT)
    assert abs(len(gpu) - len(cpu)) / len(cpu) < 0.01
    kg = (gpu["path"].astype(np.int64) << 8) | gpu["depth"]
    kc = (cpu["path"].astype(np.int64) << 8) | cpu["depth"]
    common, ig, ic = np.intersect1d(kg, kc, return_indices=True)
    assert len(common) / len(cpu) > 0.97
    close = np.all(np.abs(gpu["pos"][ig] - cpu["pos"][ic]) < 1e-3, axis=1)
    assert close.mean() > 0.97
    same_shape = gpu["shape_id"][ig] == cpu["shape_id"][ic]
    assert same_shape.mean() > 0.97
    rel = np.abs(gpu["power"][ig] - cpu["power"][ic]) / np.maximum(np.abs(cpu["power"][ic]), 1e-12)
    assert np.median(rel) < 1e-4
    # total stored power agrees
    assert abs(gpu["power"].sum() - cpu["power"].sum()) / cpu["power"].sum() < 0.02


@pytest.mark.parametrize("k", [1, 50, 128])
def test_density_estimate_matches_formula(core, gpu_ctx, restated, k):
    """Scene::combinePhotonContributions on a traced photon map: sum over the k nearest
    same-shape photons of power * kd/pi * |cos| / (pi * maxDist^2), recomputed in numpy from
    the same photons and the brute-force neighbour sets."""
    import torch

    rng = np.random.default_rng(3)
    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, 16, 16)
    sc.add_point_light((0.0, 0.9, 0.0), (1.0, 1.0, 1.0), 5.0)
    sc.commit()
    pm, _ = sc.trace_photons(100000, max_depth=30, seed=4)
    pm.build()
    photons = pm.photons()
    floor = photons[photons["shape_id"] == 0]  # the floor mesh (shape 0): y = -1
    q = floor["pos"][:300].copy()
    q[:, :2] += rng.normal(0, 0.01, (300, 2)).astype(np.float32) * np.array([1, 0], np.float32)
    nrm = np.tile(np.array([0, 1, 0], np.float32), (300, 1))
    wo = np.tile(np.array([0.3, 0.9, 0.1], np.float32) / np.linalg.norm([0.3, 0.9, 0.1]), (300, 1)).astype(np.float32)
    kd = np.array([0.8, 0.8, 0.8])
    mat = core.material(N.RT_MAT_LAMBERTIAN, color=kd)
    radius = 0.5
    qs = np.zeros(300, np.int32)
    got = pm.density(mat, torch.from_numpy(q).cuda(), torch.from_numpy(nrm).cuda(), torch.from_numpy(wo).cuda(),
                          k, radius, torch.from_numpy(qs).cuda()).cpu().numpy()
    idx, dist, cnt = restated.knn(photons["pos"], photons["shape_id"], q, qs, k, radius)
    for i in range(300):
        sel = photons[idx[i, :cnt[i]]]
        if cnt[i] == 0:
            assert np.all(got[i] == 0)
            continue
        maxd = np.sqrt(((sel["pos"] - q[i]) ** 2).sum(1)).max()
        cos = np.abs(-sel["dir"] @ nrm[i])
        exp = (sel["power"] * (kd / np.pi)[None, :] * cos[:, None]).sum(0) / (np.pi * maxd * maxd)
        assert np.allclose(got[i], exp, rtol=2e-4, atol=0), (i, got[i], exp)


def test_photon_mapping_render_agrees_with_path_tracing(core, gpu_ctx):
    """RENDER_MODE PHOTON_MAPPING (gather at the first diffuse hit) against path tracing on the
    Cornell box lit by a point light: same image mean within the photon-map blur."""
    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, 64, 64)
    sc.add_point_light((0.0, 0.8, 0.2), (1.0, 1.0, 1.0), 3.0)
    sc.set_materials(cfg.cornell_materials()[:3] + [core.material(N.RT_MAT_LAMBERTIAN, color=(0.8, 0.8, 0.8))]
                     + cfg.cornell_materials()[4:])  # the ceiling quad does not emit here
    sc.commit()
    pm, st = sc.trace_photons(2_000_000, max_depth=30, seed=2)
    pm.build()
    sc.set_photon_map(pm, k=100, radius=100.0)
    film, rst = sc.render(cam, spp=16, max_depth=8, flags=N.RT_RENDER_PHOTON_MAP, fp64=True)
    pmimg = core.film_mean(film)
    ref, _ = sc.render(cam, spp=256, max_depth=8, flags=0, fp64=True)
    ptimg = core.film_mean(ref)
    assert np.isfinite(pmimg).all()
    assert abs(pmimg.mean() - ptimg.mean()) / ptimg.mean() < 0.10
    # the reference's estimate also weights each photon by |cos| (SurfaceInteraction::lightScattered):
    # darker by the mean incidence cosine of the photons
    cf, _ = sc.render(cam, spp=16, max_depth=8, flags=N.RT_RENDER_PHOTON_MAP | N.RT_RENDER_COMPAT, fp64=True)
    ratio = core.film_mean(cf).mean() / pmimg.mean()
    assert 0.4 < ratio < 0.95


def test_config4_knn_set_against_reference_kdtree(core, gpu_ctx, refo):
    """The 4K photon-mapping configuration's gather: the photon map of 10M emitted photons over
    the 2M-triangle terrain, the subsurface slab and 16 glass spheres, and 2^20 query points on
    its surfaces with their shape ids (the stored photons of an independent trace), k = 50 nearest
    on the same shape within the reference's default radius (100, types.h:58). Every neighbour
    count equals the reference kd-tree's (nn::KDTree, kdtree.h:111-152); every neighbour set equals
    it except for members tied at the k-th distance, which the reference's heap order decides.
    The number of such tie-broken sets is reported."""
    import torch
    from oracle import bindings

    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    sc, _, _ = cfgs.build_config4(gpu_ctx, 64, 36)
    pm, st = sc.trace_photons(10_000_000, max_depth=16, seed=12)
    pm.build()
    ph = pm.photons()
    qm, _ = sc.trace_photons(6_000_000, max_depth=16, seed=99)  # about 0.2 stored per emitted photon
    qp = qm.photons()
    nq = 1 << 20
    assert len(qp) >= nq
    q, qs = np.ascontiguousarray(qp["pos"][:nq]), np.ascontiguousarray(qp["shape_id"][:nq])
    k, radius = 50, 100.0
    gi, gd, gc = pm.knn(torch.from_numpy(q.reshape(-1)).cuda(), k, radius, torch.from_numpy(qs).cuda())
    gi, gd, gc = gi.cpu().numpy(), gd.cpu().numpy(), gc.cpu().numpy()
    pos, shp = np.ascontiguousarray(ph["pos"]), np.ascontiguousarray(ph["shape_id"])
    kd = bindings.RefKdTree(refo, pos, shp)
    import os

    ri, rc = kd.knn(q, k, radius, qs, threads=os.cpu_count() or 8)
    assert np.array_equal(gc, rc.astype(np.int32))
    assert (gc == k).mean() > 0.99
    col = np.arange(k)[None, :]
    gs = np.sort(np.where(col < gc[:, None], gi, -1), axis=1)
    rs = np.sort(np.where(col < rc[:, None].astype(np.int64), ri, -1), axis=1)
    differ = np.flatnonzero(np.any(gs != rs, axis=1))
    for i in differ:
        a, b = set(gi[i, :gc[i]].tolist()), set(ri[i, :rc[i]].tolist())
        kth = gd[i, gc[i] - 1]
        dd = np.sqrt(((pos[list(a ^ b)].astype(np.float64) - q[i]) ** 2).sum(1))
        assert np.allclose(dd, kth, rtol=1e-6, atol=0), (i, dd, kth)
    print(f"config-4 k-NN: {len(ph)} photons, {nq} queries, {len(differ)} sets differ only by members tied "
          f"at the k-th distance ({len(differ) / nq:.2e})")
    assert len(differ) < 1e-3 * nq
