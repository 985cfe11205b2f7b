"""Phong surfaces and subsurface scattering (SSMaterial): the Phong BSDF of the CPU
restatement against the reference's PhongMaterial (CPU), the GPU dipole photon estimate
against the reference's diffusionTermBSSRDF over brute-force neighbour sets, and the
subsurface and hybrid render modes against identities that hold sample by sample."""
import importlib

import numpy as np
import pytest

N = importlib.import_module("2023_render_engine_b200._native")


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def test_phong_restatement_matches_reference(core, restated, refo):
    from oracle import bindings

    rng = np.random.default_rng(0)
    wo, wi = unit(rng.normal(size=(4000, 3))), unit(rng.normal(size=(4000, 3)))
    wo[:, 2] = np.abs(wo[:, 2]) * np.where(rng.uniform(size=4000) < 0.8, 1, -1)
    kd, ks, ns = (0.6, 0.3, 0.2), (0.3, 0.35, 0.4), 12.0
    f_ref, p_ref = bindings.ref_phong_eval(refo, kd, ks, ns, wo, wi)
    f, p = bindings.restated_phong_eval(restated, core.phong_material(kd, ks, ns), wo, wi)
    assert np.allclose(f, f_ref, rtol=2e-5, atol=1e-7)
    assert np.allclose(p, p_ref, rtol=2e-5, atol=1e-7)


SIG_S, SIG_A, G, ETA = (1.0, 0.8, 0.6), (0.01, 0.02, 0.05), 0.0, 1.3


def floor_scene(core, ctx, material):
    """Two 2x2 quads side by side at z = 0 (shapes 0 and 1) under a point light."""
    sc = core.Scene(ctx)
    sc.set_materials([material])
    for i, x0 in enumerate((-2.0, 0.0)):
        v = np.array([[x0, -1, 0], [x0 + 2, -1, 0], [x0 + 2, 1, 0], [x0, 1, 0]], np.float32)
        sc.add_mesh(v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), material=0, shape_id=i)
    sc.add_point_light((0.3, 0.2, 1.0), (1, 1, 1), 5.0)
    sc.commit()
    return sc


def down_camera(core, w=32, h=32):
    return core.look_at_camera((0.0, 0.0, 2.0), (0, 0, 0), (0, 1, 0), 50.0, w, h)


@pytest.mark.gpu
def test_dipole_estimate_matches_reference(core, gpu_ctx, refo):
    import torch
    from oracle import bindings

    mat = core.subsurface_material((0.9, 0.8, 0.7), (0, 0, 0), 1.0, ETA, SIG_S, SIG_A, G)
    sc = floor_scene(core, gpu_ctx, mat)
    pm, _ = sc.trace_photons(20000, max_depth=1, seed=3)
    pm.build()
    ph = pm.photons()
    assert len(ph) > 2000
    rng = np.random.default_rng(1)
    nq = 40
    q = np.concatenate([rng.uniform(-1.5, 1.5, (nq, 1)), rng.uniform(-0.8, 0.8, (nq, 1)), np.zeros((nq, 1))],
                       1).astype(np.float32)
    qn = np.tile(np.array([0, 0, 1], np.float32), (nq, 1))
    wo = unit(rng.normal(size=(nq, 3)) + np.array([0, 0, 2.0])).astype(np.float32)
    qs = (q[:, 0] >= 0).astype(np.int32)
    out = torch.empty(nq * 3, dtype=torch.float32, device="cuda")
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    args = [cu(a) for a in (q, qn, wo, qs)]  # held until the call returns
    N.check(N.lib().rt_photon_subsurface(pm.handle, ctypes_byref(mat), *[a.data_ptr() for a in args], nq, 0.3, 0,
                                         out.data_ptr()))
    got = out.cpu().numpy().reshape(nq, 3)
    P = ph["pos"].astype(np.float64)
    kd = np.array(mat.color, np.float64)
    for i in range(nq):
        d = np.sqrt(((P - q[i]) ** 2).sum(1))
        sel = np.nonzero((d < 0.3) & (ph["shape_id"] == qs[i]))[0]
        assert len(sel) > 20
        acc = np.zeros(3)
        for j in sel:
            sd = bindings.ref_diffusion_term(refo, q[i], wo[i], qn[i], ph["pos"][j], ph["dir"][j], ph["normal"][j],
                                             SIG_S, SIG_A, G, ETA)
            acc += sd * ph["power"][j] * kd
        want = acc / (2 * np.pi * d[sel].max() ** 2)
        assert np.allclose(got[i], want, rtol=2e-4, atol=1e-12), (i, got[i], want)


@pytest.mark.gpu
def test_subsurface_mode_adds_the_dipole_estimate_at_camera_hits(core, gpu_ctx):
    """Depth 1 renders with and without RT_RENDER_SUBSURFACE share every sample; their
    difference is the dipole estimate at the primary hits, which is smooth across a pixel."""
    import torch

    mat = core.subsurface_material((0.9, 0.8, 0.7), (0, 0, 0), 1.0, ETA, SIG_S, SIG_A, G)
    sc = floor_scene(core, gpu_ctx, mat)
    pm, _ = sc.trace_photons(200000, max_depth=1, seed=4)
    pm.build()
    sc.set_photon_map(pm, 50, 1.0)
    cam = down_camera(core)
    fa, _ = sc.render(cam, spp=64, max_depth=1, seed=5, flags=N.RT_RENDER_SUBSURFACE, fp64=True)
    fb, _ = sc.render(cam, spp=64, max_depth=1, seed=5, flags=0, fp64=True)
    diff = (core.film_mean(fa) - core.film_mean(fb)).reshape(32, 32, 3)
    # the estimate at the pixel centres (the hit points of the centre rays on z = 0)
    ys, xs = np.mgrid[0:32, 0:32]
    r2c = np.array(cam.raster_to_camera).reshape(4, 4)
    c2w = np.array(cam.camera_to_world).reshape(4, 4)
    pts = np.stack([xs.ravel() + 0.5, ys.ravel() + 0.5, np.zeros(1024), np.ones(1024)], 1) @ r2c.T
    dc = pts[:, :3] / pts[:, 3:]
    dw = unit(dc @ c2w[:3, :3].T)
    eye = c2w[:3, 3]
    hit = eye + dw * (-eye[2] / dw[:, 2:3])
    q = hit.astype(np.float32)
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    out = torch.empty(1024 * 3, dtype=torch.float32, device="cuda")
    args = [cu(a) for a in (q, np.tile([0, 0, 1], (1024, 1)).astype(np.float32), (-dw).astype(np.float32),
                            (q[:, 0] >= 0).astype(np.int32))]  # held until the call returns
    N.check(N.lib().rt_photon_subsurface(pm.handle, ctypes_byref(mat), *[a.data_ptr() for a in args], 1024, 0.3, 0,
                                         out.data_ptr()))
    want = out.cpu().numpy().reshape(32, 32, 3)
    inner = np.abs(q[:, 0].reshape(32, 32)) > 0.4  # away from the seam between the two shapes
    inner &= (np.abs(q[:, 0]) < 1.6).reshape(32, 32) & (np.abs(q[:, 1]) < 0.7).reshape(32, 32)
    assert inner.sum() > 100
    rel = np.abs(diff[inner] - want[inner]).max(1) / want[inner].max(1)
    assert np.median(rel) < 0.02 and rel.max() < 0.1


@pytest.mark.gpu
def test_hybrid_mode_is_the_mean_of_photon_density_and_next_event(core, gpu_ctx):
    """At depth 1 (no emitters) the hybrid direct term (density + NEE) / 2 equals the mean of
    the photon-mapping render and the path-traced render with the same samples."""
    sc = floor_scene(core, gpu_ctx, core.material(N.RT_MAT_LAMBERTIAN, color=(0.7, 0.6, 0.5)))
    pm, _ = sc.trace_photons(100000, max_depth=4, seed=6)
    pm.build()
    sc.set_photon_map(pm, 50, 1.0)
    cam = down_camera(core)
    fh, _ = sc.render(cam, spp=16, max_depth=1, seed=7, flags=N.RT_RENDER_HYBRID, fp64=True)
    fp, _ = sc.render(cam, spp=16, max_depth=1, seed=7, flags=N.RT_RENDER_PHOTON_MAP, fp64=True)
    fn, _ = sc.render(cam, spp=16, max_depth=1, seed=7, flags=0, fp64=True)
    h, p, n = core.film_mean(fh), core.film_mean(fp), core.film_mean(fn)
    assert np.allclose(h, (p + n) / 2, rtol=1e-4, atol=1e-7)
    assert p.mean() > 0 and n.mean() > 0


def covered_floor_scene(core, ctx):
    """floor_scene with a 4x2 ceiling quad at z = 1.6 (shape 2) that paths bounce back from."""
    sc = core.Scene(ctx)
    sc.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=(0.7, 0.6, 0.5))])
    quads = [np.array([[x0, -1, 0], [x0 + 2, -1, 0], [x0 + 2, 1, 0], [x0, 1, 0]], np.float32) for x0 in (-2.0, 0.0)]
    quads.append(np.array([[-2, -1, 1.6], [-2, 1, 1.6], [2, 1, 1.6], [2, -1, 1.6]], np.float32))
    for i, v in enumerate(quads):
        sc.add_mesh(v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), material=0, shape_id=i)
    sc.add_point_light((0.3, 0.2, 1.0), (1, 1, 1), 5.0)
    sc.commit()
    return sc


@pytest.mark.gpu
def test_guide_records_take_the_hybrid_photon_estimates(core, gpu_ctx):
    """With the same samples, the guide records of a hybrid render hold half the next-event
    radiance of a plain render plus half the photon density estimates: strictly more than
    half, which they would be if the gathers did not reach the records."""
    sc = covered_floor_scene(core, gpu_ctx)
    pm, _ = sc.trace_photons(100000, max_depth=4, seed=6)
    pm.build()
    sc.set_photon_map(pm, 50, 1.0)
    cam = core.look_at_camera((0.0, 0.0, 1.4), (0, 0, 0), (0, 1, 0), 70.0, 32, 32)
    g = core.Guide(gpu_ctx, (-2.1, -1.1, -0.1), (2.1, 1.1, 1.7), learning_rate=1e-3, seed=1, max_depth=3)
    sums = {}
    for name, fl in (("plain", 0), ("hybrid", N.RT_RENDER_HYBRID)):
        sc.set_guide(g, train=True)
        sc.render(cam, spp=4, max_depth=4, seed=9, flags=fl | N.RT_RENDER_GUIDE)
        r = g.records()
        assert len(r) > 1000
        sums[name] = r[:, 16:19].astype(np.float64).sum(0)
    sc.set_guide(None)
    g.close()
    assert np.all(sums["plain"] > 0)
    assert np.all(sums["hybrid"] > 0.5 * sums["plain"] * 1.05), sums


@pytest.mark.gpu
def test_guided_hybrid_subsurface_render_is_unbiased(core, gpu_ctx):
    """A guide trained on hybrid + subsurface renders (its records hold the photon estimates)
    leaves the image mean unchanged: one-sample MIS keeps the estimator unbiased."""
    import torch

    sc = covered_floor_scene(core, gpu_ctx)
    pm, _ = sc.trace_photons(100000, max_depth=4, seed=6)
    pm.build()
    sc.set_photon_map(pm, 50, 1.0)
    cam = core.look_at_camera((0.0, 0.0, 1.4), (0, 0, 0), (0, 1, 0), 70.0, 32, 32)
    fl = N.RT_RENDER_HYBRID | N.RT_RENDER_SUBSURFACE
    g = core.Guide(gpu_ctx, (-2.1, -1.1, -0.1), (2.1, 1.1, 1.7), learning_rate=1e-3, seed=1, max_depth=3)
    for i in range(3):
        sc.set_guide(g, train=True)
        sc.render(cam, spp=4, max_depth=6, seed=20 + i, flags=fl | N.RT_RENDER_GUIDE)
        assert g.record_count()[1] > 0
        g.train_records(32, 1 << 14, seed=i)
    sc.set_guide(g, train=False)
    fg, _ = sc.render(cam, spp=1024, max_depth=6, seed=31, flags=fl | N.RT_RENDER_GUIDE, fp64=True)
    fp, _ = sc.render(cam, spp=1024, max_depth=6, seed=32, flags=fl, fp64=True)
    torch.cuda.synchronize()
    mg, mp = core.film_mean(fg).mean(0), core.film_mean(fp).mean(0)
    assert np.all(np.isfinite(mg)) and np.all(mp > 0)
    assert np.allclose(mg, mp, rtol=0.02), (mg, mp)
    with pytest.raises(N.RtError):
        sc.render(cam, spp=1, max_depth=2, seed=1, flags=N.RT_RENDER_PHOTON_MAP | N.RT_RENDER_GUIDE)
    sc.set_guide(None)
    g.close()


def ctypes_byref(x):
    import ctypes

    return ctypes.byref(x)
