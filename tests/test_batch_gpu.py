"""Batched rendering (rt_render_batch): many views of one scene in one wavefront. Each view
renders exactly the samples rt_render gives it with the same options, so a batched view
equals its own render up to the order of the film's float atomics."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
C = importlib.import_module("2023_render_engine_b200.configs")


def views_cornell(core):
    cams = [core.look_at_camera((0, 0, 3.5), (0, 0, 0), (0, 1, 0), 40.0, 48, 32),
            core.look_at_camera((0.3, 0.2, 2.5), (0, -0.3, 0), (0, 1, 0), 55.0, 17, 29),
            core.look_at_camera((-0.5, 0.5, 3.0), (0.2, -0.5, 0), (0, 1, 0), 35.0, 64, 64)]
    return [dict(camera=cams[0], spp=4, max_depth=8, rr_depth=3, seed=1),
            dict(camera=cams[1], spp=16, max_depth=12, rr_depth=3, seed=2, sample_offset=5),
            dict(camera=cams[2], spp=2, max_depth=5, rr_depth=2, seed=3)]


@pytest.mark.parametrize("flags", [N.RT_RENDER_NEE_AREA, N.RT_RENDER_COMPAT])
def test_batch_views_equal_their_own_renders(core, gpu_ctx, flags):
    sc, _, _ = C.build_config0(gpu_ctx, 16, 16)
    views = views_cornell(core)
    film, st, off = sc.render_batch(views, flags=flags, fp64=True)
    s64 = film["sum64"].cpu().numpy().reshape(-1, 3)
    cnt = film["count"].cpu().numpy()
    total_ext = 0
    for i, v in enumerate(views):
        f1, st1 = sc.render(v["camera"], spp=v["spp"], max_depth=v["max_depth"], rr_depth=v["rr_depth"],
                            seed=v["seed"], sample_offset=v.get("sample_offset", 0), flags=flags, fp64=True)
        total_ext += st1["extension_rays"]
        a = s64[off[i]:off[i + 1]]
        b = f1["sum64"].cpu().numpy().reshape(-1, 3)
        assert np.array_equal(cnt[off[i]:off[i + 1]], f1["count"].cpu().numpy())
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6), i
    assert st["extension_rays"] == total_ext
    assert st["camera_rays"] == sum(v["camera"].width * v["camera"].height * v["spp"] for v in views)


def test_single_view_batch_is_rt_render(core, gpu_ctx):
    sc, cam, p = C.build_config0(gpu_ctx, 40, 30)
    film, st, _ = sc.render_batch([dict(camera=cam, spp=8, max_depth=8, seed=4)], flags=N.RT_RENDER_NEE_AREA,
                                  fp64=True)
    f1, st1 = sc.render(cam, spp=8, max_depth=8, seed=4, flags=N.RT_RENDER_NEE_AREA, fp64=True)
    assert np.array_equal(film["count"].cpu().numpy(), f1["count"].cpu().numpy())
    assert np.allclose(film["sum64"].cpu().numpy(), f1["sum64"].cpu().numpy(), rtol=1e-5, atol=1e-6)
    assert st["extension_rays"] == st1["extension_rays"] and st["shadow_rays"] == st1["shadow_rays"]


def test_many_waves_replay_the_captured_group(core, gpu_ctx):
    """A small queue forces many 4-wave groups (the second is captured as a CUDA graph and
    replayed): the image is the same as with a queue that finishes in few groups."""
    sc, cam, p = C.build_config0(gpu_ctx, 32, 32)
    f_small, st_small = sc.render(cam, spp=16, max_depth=8, seed=9, flags=N.RT_RENDER_NEE_AREA, fp64=True,
                                  max_paths=1024)
    f_big, st_big = sc.render(cam, spp=16, max_depth=8, seed=9, flags=N.RT_RENDER_NEE_AREA, fp64=True)
    assert st_small["waves"] > 8 * st_big["waves"]
    assert np.array_equal(f_small["count"].cpu().numpy(), f_big["count"].cpu().numpy())
    assert np.allclose(f_small["sum64"].cpu().numpy(), f_big["sum64"].cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_batch_rejects_bad_views(core, gpu_ctx):
    sc, cam, _ = C.build_config0(gpu_ctx, 8, 8)
    with pytest.raises(Exception):
        sc.render_batch([dict(camera=cam, spp=0)])
    with pytest.raises(Exception):
        sc.render_batch([])


def _textured_floor(core, ctx):
    """A textured Lambertian quad under a point light and a quad emitter (texture ids, uvs and
    point lights of a scene that is not the first of a merge)."""
    sc = core.Scene(ctx)
    tex = np.random.default_rng(1).uniform(0.1, 1.0, (4, 4, 3)).astype(np.float32)
    tid = sc.add_texture(tex)
    sc.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=(0.9, 0.8, 0.7), texture=tid),
                      core.material(N.RT_MAT_LIGHT, color=(1, 1, 1), intensity=8.0)])
    floor = np.array([[-2, 0, -2], [2, 0, -2], [2, 0, 2], [-2, 0, 2]], np.float32)
    light = np.array([[-0.5, 1.5, -0.5], [-0.5, 1.5, 0.5], [0.5, 1.5, 0.5], [0.5, 1.5, -0.5]], np.float32)
    q = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)
    first = sc.add_mesh(floor, q, material=0, shape_id=0)
    sc.set_triangle_uvs(first, np.array([[0, 0, 1, 1, 1, 0], [0, 0, 0, 1, 1, 1]], np.float32))
    sc.add_mesh(light, q, material=1, shape_id=1)
    sc.add_point_light((0.5, 1.0, 0.5), (1, 0.9, 0.8), 2.0)
    sc.commit()
    return sc


def test_merged_scenes_render_like_each_scene(core, gpu_ctx):
    """rt_scene_merge: views of three scenes (the Cornell box with its spheres and area light, a
    small BVH-stress mesh with per-block GGX, a textured floor with a point light) in one
    wavefront give every view the image rt_render_batch of its own scene gives it."""
    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    s0, cam0, _ = cfgs.build_config0(gpu_ctx, 40, 32)
    s1, cam1, _ = cfgs.build_config1(gpu_ctx, 48, 24, subdiv=3)
    s2 = _textured_floor(core, gpu_ctx)
    cam2 = core.look_at_camera((0, 1.2, 3.0), (0, 0, 0), (0, 1, 0), 50.0, 32, 32)
    per_scene = [(s0, [dict(camera=cam0, spp=4, max_depth=8, seed=1), dict(camera=cam0, spp=2, max_depth=5, seed=2)]),
                 (s1, [dict(camera=cam1, spp=3, max_depth=12, seed=3)]),
                 (s2, [dict(camera=cam2, spp=4, max_depth=6, seed=4), dict(camera=cam2, spp=1, max_depth=3, seed=5)])]
    flags = N.RT_RENDER_NEE_AREA
    want, rays = [], 0
    for sc, views in per_scene:
        film, st, off = sc.render_batch(views, flags=flags, fp64=True, max_paths=1 << 14)
        m = core.film_mean(film)
        want += [m[off[i]:off[i + 1]] for i in range(len(views))]
        rays += st["extension_rays"] + st["shadow_rays"]
    merged = core.merge_scenes(gpu_ctx, [s0, s1, s2])
    views = [dict(v, scene=k) for k, (_, vs) in enumerate(per_scene) for v in vs]
    film, st, off = merged.render_batch(views, flags=flags, fp64=True, max_paths=1 << 14)
    m = core.film_mean(film)
    assert st["extension_rays"] + st["shadow_rays"] == rays
    for i in range(len(views)):
        assert np.allclose(m[off[i]:off[i + 1]], want[i], rtol=1e-5, atol=1e-6), i
    with pytest.raises(N.RtError):  # a merged scene is not traced or modified
        merged.add_point_light((0, 0, 0), (1, 1, 1), 1.0)
    with pytest.raises(N.RtError):
        merged.render_batch([dict(camera=cam0, spp=1, scene=3)])
    merged.close()
