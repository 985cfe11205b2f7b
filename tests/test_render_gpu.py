"""Path-tracer checks through the C ABI: analytic scenes (exact answers) and the
Cornell box against the C restatement of the estimator."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
S = importlib.import_module("2023_render_engine_b200.scenes")


def quad_mesh(z, half, flip=False):
    v = np.array([[-half, -half, z], [half, -half, z], [half, half, z], [-half, half, z]], np.float32)
    f = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    if flip:
        f = f[:, ::-1].copy()
    return v, f


def test_emitter_seen_directly(core, gpu_ctx):
    """Every camera sample hits a Le = (2, 3, 4) emitter: each pixel equals Le exactly."""
    sc = core.Scene(gpu_ctx)
    sc.set_materials([core.material(N.RT_MAT_LIGHT, color=(2, 3, 4), intensity=1.0)])
    v, f = quad_mesh(-2.0, 50.0)
    sc.add_mesh(v, f, material=0)
    sc.commit()
    cam = core.look_at_camera((0, 0, 0), (0, 0, -1), (0, 1, 0), 40.0, 32, 24)
    film, st = sc.render(cam, spp=4, max_depth=4)
    img = core.film_mean(film)
    assert np.allclose(img, [2, 3, 4])
    assert film["count"].cpu().numpy().min() == 4
    assert st["camera_rays"] == 32 * 24 * 4
    assert st["extension_rays"] == 32 * 24 * 4


@pytest.mark.parametrize("compat", [False, True])
def test_point_light_on_lambertian_floor(core, gpu_ctx, compat):
    """Direct light only (bounces escape): L = kd/pi * cos * I / d^2; the reference's
    delta-light MIS weight 1/(1 + pdf^2) (Scene.cu:331) scales it in compat mode."""
    kd = np.array([0.5, 0.6, 0.7])
    sc = core.Scene(gpu_ctx)
    sc.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=kd)])
    v, f = quad_mesh(0.0, 100.0)
    sc.add_mesh(v, f, material=0)
    lp = np.array([0.3, -0.2, 1.0])
    sc.add_point_light(lp, (1.0, 1.0, 1.0), 2.0)
    sc.commit()
    W = H = 16
    cam = core.look_at_camera((0, 0, 3.0), (0, 0, 0), (0, 1, 0), 30.0, W, H)
    flags = N.RT_RENDER_COMPAT if compat else 0
    film, st = sc.render(cam, spp=256, max_depth=1, fp64=True, flags=flags)
    img = core.film_mean(film).reshape(H, W, 3)
    # analytic value at pixel centres (the estimate averages the pixel footprint)
    c2w = np.array(cam.camera_to_world).reshape(4, 4)
    r2c = np.array(cam.raster_to_camera).reshape(4, 4)
    exp = np.zeros((H, W, 3))
    for y in range(H):
        for x in range(W):
            pc = r2c @ np.array([x + 0.5, y + 0.5, 0, 1.0])
            dc = pc[:3] / pc[3]
            d = c2w[:3, :3] @ (dc / np.linalg.norm(dc))
            o = c2w[:3, 3]
            t = -o[2] / d[2]
            p = o + t * d
            tol = lp - p
            dist2 = tol @ tol
            cos = tol[2] / np.sqrt(dist2)
            val = kd / np.pi * cos * 2.0 / dist2
            if compat:
                val = val / (1 + (cos / np.pi) ** 2)
            exp[y, x] = val
    rel = np.abs(img - exp) / exp
    assert np.median(rel) < 0.01
    assert rel.max() < 0.05
    assert st["shadow_rays"] > 0


def test_cornell_box_renders(core, gpu_ctx):
    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, 64, 64)
    film, st = sc.render(cam, spp=8, max_depth=p["max_depth"], rr_depth=p["rr_depth"], flags=N.RT_RENDER_COMPAT)
    img = core.film_mean(film)
    assert np.isfinite(img).all()
    assert (film["count"].cpu().numpy() == 8).mean() > 0.99
    assert 0.05 < img.mean() < 5.0
    # NEE on the area light changes the variance, not the expectation
    f2, st2 = sc.render(cam, spp=64, max_depth=p["max_depth"], rr_depth=p["rr_depth"], flags=N.RT_RENDER_NEE_AREA)
    f3, _ = sc.render(cam, spp=64, max_depth=p["max_depth"], rr_depth=p["rr_depth"], flags=0, seed=5)
    a, b = core.film_mean(f2).mean(), core.film_mean(f3).mean()
    assert abs(a - b) / b < 0.03
    assert st2["shadow_rays"] > 0


def _cornell_oracle(cfg, restated):
    from oracle import bindings

    sc_data = S.cornell_box()
    v, f, m = S.flatten(sc_data)
    spheres = []
    for s in sc_data["spheres"]:
        o2w, w2o = S.sphere_matrices(s["center"], s["radius"])
        spheres.append({"o2w": o2w, "w2o": w2o, "radius": s["radius"], "material": s["material"]})
    return bindings.PathTracerOracle(restated, v, f, m, spheres, cfg.cornell_materials())


@pytest.mark.parametrize("flags", [N.RT_RENDER_COMPAT, N.RT_RENDER_NEE_AREA])
def test_cornell_matches_cpu_restatement(core, gpu_ctx, restated, flags):
    """Same PCG streams on both sides: per-pixel agreement up to float rounding (a few
    paths diverge where rounding flips a decision), and matching image means."""
    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, 48, 48)
    film, _ = sc.render(cam, spp=8, max_depth=p["max_depth"], rr_depth=p["rr_depth"], flags=flags, fp64=True, seed=3)
    gpu = core.film_mean(film)
    orc = _cornell_oracle(cfg, restated)
    s, c = orc.render(cam, spp=8, max_depth=p["max_depth"], rr_depth=p["rr_depth"], flags=flags, seed=3)
    cpu = s / np.maximum(c, 1)[:, None]
    assert np.array_equal(film["count"].cpu().numpy(), c.astype(np.int32))
    rel = np.abs(gpu - cpu).max(axis=1) / np.maximum(np.abs(cpu).max(axis=1), 1e-6)
    assert np.median(rel) < 1e-4
    assert (rel < 1e-3).mean() > 0.8
    assert abs(gpu.mean() - cpu.mean()) / cpu.mean() < 0.02


@pytest.mark.parametrize("log2", [5, 9, 13])
def test_material_sort_leaves_the_image_unchanged(core, gpu_ctx, log2):
    """The material sort only reorders which thread shades which path: every path keeps its own
    random stream, so the image equals the unsorted one up to the order of film additions."""
    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfgs.build_config0(gpu_ctx, 64, 64)
    sc.add_point_light((0.0, 0.5, 0.0), (1.0, 1.0, 1.0), 2.0)
    sc.commit()
    flags = N.RT_RENDER_NEE_AREA
    ref, st0 = sc.render(cam, spp=8, max_depth=8, seed=3, flags=flags, fp64=True, max_paths=1 << 14)
    sc.set_sort(log2)
    got, st1 = sc.render(cam, spp=8, max_depth=8, seed=3, flags=flags, fp64=True, max_paths=1 << 14)
    sc.set_sort(0)
    a, b = core.film_mean(ref), core.film_mean(got)
    assert st0["extension_rays"] == st1["extension_rays"] and st0["shadow_rays"] == st1["shadow_rays"]
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
    with pytest.raises(N.RtError):
        sc.set_sort(20)


def test_device_wave_loop_equals_host_loop(core, gpu_ctx):
    """On a stream of its own a render runs its waves as one CUDA graph with a conditional WHILE
    node ended on the device; on the legacy default stream (which cannot be captured) the host
    checks after every 4-wave group. Both render the same samples: equal ray counts and images."""
    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    out = []
    for legacy in (False, True):
        ctx = core.Context(0)
        if legacy:
            ctx.set_stream(0)
        sc, cam, p = cfgs.build_config0(ctx, 48, 48)
        film, st = sc.render(cam, spp=8, max_depth=8, seed=11, flags=N.RT_RENDER_NEE_AREA, fp64=True,
                             max_paths=1 << 12)  # small queues: many wave groups
        out.append((core.film_mean(film), st))
        sc.close()
    (a, sa), (b, sb) = out
    assert sa["extension_rays"] == sb["extension_rays"] and sa["shadow_rays"] == sb["shadow_rays"]
    assert sa["waves"] == sb["waves"] and sa["waves"] > 8
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_path_capacity_leaves_the_image_unchanged(core, gpu_ctx):
    """The capacity (paths in flight) only decides how many waves a frame takes: every sample
    keeps its own random stream, so small queues, the automatic capacity (max_paths 0: here
    all of the frame's samples at once) and a capacity above the samples give the same rays
    and the same image up to the order of film additions; the retire and sort kernels'
    grid-stride loops see from one to many chunks per block."""
    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfgs.build_config0(gpu_ctx, 64, 48)
    flags = N.RT_RENDER_NEE_AREA
    out = []
    for cap in (1 << 10, 0, 1 << 20):
        film, st = sc.render(cam, spp=6, max_depth=8, seed=5, flags=flags, fp64=True, max_paths=cap)
        out.append((core.film_mean(film), st))
    (a, sa) = out[0]
    assert sa["waves"] > out[1][1]["waves"]
    for b, sb in out[1:]:
        assert sa["extension_rays"] == sb["extension_rays"] and sa["shadow_rays"] == sb["shadow_rays"]
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


def test_stage_times(core, gpu_ctx):
    """RT_RENDER_STAGE_TIMES times every wavefront stage with CUDA events (host loop, no graphs):
    the same samples as an untimed render, a time for each stage that ran, none for the stages
    that did not (no guide, no photon map), and a sum within the call's own time."""
    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfgs.build_config0(gpu_ctx, 64, 48)
    flags = N.RT_RENDER_NEE_AREA
    ref, st0 = sc.render(cam, spp=4, max_depth=8, seed=9, flags=flags, fp64=True, max_paths=1 << 12)
    assert all(v == 0.0 for v in sc.stage_times().values())
    got, st1 = sc.render(cam, spp=4, max_depth=8, seed=9, flags=flags | N.RT_RENDER_STAGE_TIMES, fp64=True,
                         max_paths=1 << 12)
    t = sc.stage_times()
    assert st0["extension_rays"] == st1["extension_rays"] and st0["shadow_rays"] == st1["shadow_rays"]
    assert np.allclose(core.film_mean(ref), core.film_mean(got), rtol=1e-5, atol=1e-6)
    for k in ("trace", "material_sort", "shade", "shadow", "retire"):
        assert t[k] > 0.0
    # nothing runs between those two pairs of events: only the events' own spacing is timed
    assert t["gather"] < 0.25 * t["trace"] and t["guide_inference"] < 0.25 * t["trace"]
    assert sum(t.values()) <= st1["ms"] * 1.001
    # an untimed render clears them again
    sc.render(cam, spp=1, max_depth=8, seed=9, flags=flags)
    assert all(v == 0.0 for v in sc.stage_times().values())
    with pytest.raises(N.RtError):
        N.check(N.lib().rt_render_stage_times(sc.handle, None, 1))
