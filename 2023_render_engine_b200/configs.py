"""The benchmark configurations as ready-to-render scenes (geometry from scenes.py,
materials and cameras per the configuration descriptions).

* config0: Cornell box — walls 0.8 / red / green Lambertian, 0.5x0.5 ceiling light of
  emission 15, Lambertian sphere (0.8) and glass sphere (IOR 1.5), pinhole camera at
  (0,0,3.5) looking down -z with a 40 degree vertical field of view; 256x256, 16 spp,
  max depth 8, Russian roulette after depth 3.
* config1: BVH stress — the 1.31M-triangle displaced icosphere (GGX, F0 = 0.04 i.e.
  eta = 1.5, k = 0, roughness uniform in [0.05, 0.5] per block of 64 triangles) in the
  Cornell box; 1920x1080, 64 spp, max depth 12, NEE on the area light.
* config2: the guiding room; config3: 64 seeded views of configs 0-2.
* config4: photon mapping + subsurface scattering at 4K — the 2M-triangle displaced terrain,
  16 glass spheres (IOR 1.5, radius 0.1-0.4), a subsurface slab (sigma_a = (0.01, 0.02, 0.05),
  sigma_s = (1.0, 0.8, 0.6), g = 0), two point lights of 50 RGB; 10M photons, k = 50
  nearest-photon gathers; 3840x2160, 256 spp, max depth 16.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from . import core, scenes

CORNELL_MATERIALS = {
    scenes.MAT_WHITE: dict(type_=N.RT_MAT_LAMBERTIAN, color=(0.8, 0.8, 0.8)),
    scenes.MAT_RED: dict(type_=N.RT_MAT_LAMBERTIAN, color=(0.8, 0.1, 0.1)),
    scenes.MAT_GREEN: dict(type_=N.RT_MAT_LAMBERTIAN, color=(0.1, 0.8, 0.1)),
    scenes.MAT_LIGHT: dict(type_=N.RT_MAT_LIGHT, color=(1.0, 1.0, 1.0), intensity=15.0),
    scenes.MAT_DIFFUSE_SPHERE: dict(type_=N.RT_MAT_LAMBERTIAN, color=(0.8, 0.8, 0.8)),
    scenes.MAT_GLASS: dict(type_=N.RT_MAT_DIELECTRIC, color=(1.0, 1.0, 1.0), ior=1.5, transparent=True),
    scenes.MAT_GGX: dict(type_=N.RT_MAT_TROWBRIDGE, color=(1.0, 1.0, 1.0), eta=(1.5, 1.5, 1.5), k=(0, 0, 0),
                         roughness=(0.25, 0.25)),
}


def cornell_materials(extra=()):
    mats = [core.material(**CORNELL_MATERIALS[i]) for i in range(len(CORNELL_MATERIALS))]
    return mats + list(extra)


def cornell_camera(width=256, height=256):
    return core.look_at_camera((0, 0, 3.5), (0, 0, 0), (0, 1, 0), 40.0, width, height)


def build_config0(ctx, width=256, height=256):
    sc_data = scenes.cornell_box()
    sc = core.Scene(ctx)
    sc.set_materials(cornell_materials())
    for i, (v, f, m) in enumerate(sc_data["meshes"]):
        sc.add_mesh(v, f, material=m, shape_id=i)
    for j, s in enumerate(sc_data["spheres"]):
        o2w, w2o = scenes.sphere_matrices(s["center"], s["radius"])
        sc.add_sphere(o2w, w2o, s["radius"], material=s["material"], shape_id=100 + j)
    sc.commit()
    return sc, cornell_camera(width, height), dict(spp=16, max_depth=8, rr_depth=3)


def build_config1(ctx, width=1920, height=1080, subdiv=8):
    sc_data = scenes.stress_scene(subdiv=subdiv)
    rough = sc_data["roughness"]
    nblocks = (rough.shape[0] + 63) // 64
    block_r = rough[::64][:nblocks]
    extra = [core.material(N.RT_MAT_TROWBRIDGE, color=(1, 1, 1), eta=(1.5, 1.5, 1.5), k=(0, 0, 0),
                           roughness=(float(r), float(r))) for r in block_r]
    base = len(CORNELL_MATERIALS)
    sc = core.Scene(ctx)
    sc.set_materials(cornell_materials(extra))
    first = None
    for i, (v, f, m) in enumerate(sc_data["meshes"]):
        t0 = sc.add_mesh(v, f, material=m, shape_id=i)
        if m == scenes.MAT_GGX:
            first = t0
            ids = base + (np.arange(f.shape[0]) // 64)
            sc.set_triangle_materials(first, ids.astype(np.uint32))
    sc.commit()
    return sc, cornell_camera(width, height), dict(spp=64, max_depth=12, rr_depth=3)


def build_config2(ctx, width=1280, height=720, seed=3, target_triangles=200_000):
    """Config 2: the guiding room (mostly indirect light through a gap in a wall)."""
    meshes, mats = scenes.guiding_room(seed=seed, target_triangles=target_triangles)
    table = []
    for m in mats:
        if m["kind"] == "lambert":
            table.append(core.material(N.RT_MAT_LAMBERTIAN, color=m["albedo"]))
        elif m["kind"] == "ggx":
            table.append(core.material(N.RT_MAT_TROWBRIDGE, color=(1, 1, 1), eta=(1.5, 1.5, 1.5), k=(0, 0, 0),
                                       roughness=(m["roughness"], m["roughness"])))
        else:
            table.append(core.material(N.RT_MAT_LIGHT, color=m["emission"], intensity=1.0))
    sc = core.Scene(ctx)
    sc.set_materials(table)
    for i, (v, f, mi) in enumerate(meshes):
        sc.add_mesh(v, f, material=mi, shape_id=i)
    sc.commit()
    # in front of the wall, looking away from it: the emitter and the surfaces it lights
    # directly behind the wall are out of view, so the image is lit through the gap only
    cam = core.look_at_camera((0.25, 1.3, 0.75), (-0.8, 0.5, -1.6), (0, 1, 0), 65.0, width, height)
    return sc, cam, dict(spp=64, max_depth=16, rr_depth=3)


# Online training of the config-2 guide. The configuration's Adam step of 1e-2 saturates the
# sigmoid-parametrised outputs within a few dozen steps on this network (measured: alpha pinned
# at its floor, every concentration at exp(-4)); 1e-3 trains stably.
# Schedule (measured on the 1280x720 room): 4 one-spp recording passes with 128 steps each,
# guiding the first 2 bounces of every path (deeper vertices carry little of the variance and
# their inference costs as much as the shallow ones). A step's batch is one round of the
# training kernel's tiles on a 148-SM B200 (2 tiles of 128 samples per SM): 37,888 samples take
# 0.20 ms a step, 2^16 take 0.30 ms (two rounds). Time to RMSE 0.01 (median of 5), s: 0.618 for
# 64 steps of 2^16, 0.585 for 64 of 37,888, 0.570-0.585 for 128 of 37,888, 0.610 for 192, 0.665
# for 256, 0.616-0.618 for 256 of 2^14 or 18,944; plain 0.740-0.745.
GUIDE_BATCH = 2 * 148 * 128
GUIDE_TRAINING = dict(learning_rate=1e-3, batch=GUIDE_BATCH, train_passes=4, steps_per_pass=128, max_depth=2,
                      bbox_min=(-2.01, -0.01, -2.01), bbox_max=(2.01, 2.51, 2.01))


def random_views(rng, n, eye_lo, eye_hi, target_lo, target_hi, max_depth_range=(8, 16)):
    """n seeded views: eye uniform in a box, looking at a point uniform in another box;
    resolution log-uniform in [128^2, 1024^2] pixels with aspect ratio in [0.5, 2];
    spp in {4, 8, 16, 32, 64}; max depth uniform in max_depth_range."""
    views = []
    for _ in range(n):
        eye = rng.uniform(eye_lo, eye_hi)
        target = rng.uniform(target_lo, target_hi)
        area = float(np.exp(rng.uniform(np.log(128 * 128), np.log(1024 * 1024))))
        aspect = float(rng.uniform(0.5, 2.0))
        w = int(np.clip(round(np.sqrt(area * aspect)), 16, 2048))
        h = int(np.clip(round(np.sqrt(area / aspect)), 16, 2048))
        cam = core.look_at_camera(tuple(eye), tuple(target), (0, 1, 0), float(rng.uniform(35, 70)), w, h)
        views.append(dict(camera=cam, spp=int(rng.choice([4, 8, 16, 32, 64])),
                          max_depth=int(rng.integers(max_depth_range[0], max_depth_range[1] + 1)), rr_depth=3,
                          seed=int(rng.integers(0, 2 ** 31))))
    return views


def build_config3(ctx, n_views=64, seed=5):
    """Config 3: n_views instances drawn from configs 0-2 with seeded camera poses,
    resolutions, spp and depths. Returns [(name, scene, flags, views)], one entry per scene
    (each is one rt_render_batch call)."""
    rng = np.random.default_rng(seed)
    counts = np.bincount(rng.integers(0, 3, n_views), minlength=3)
    out = []
    sc0, _, _ = build_config0(ctx, 16, 16)
    out.append(("config 0 (Cornell box)", sc0, N.RT_RENDER_NEE_AREA,
                random_views(rng, int(counts[0]), (-0.6, -0.6, 2.0), (0.6, 0.6, 4.0), (-0.4, -0.6, -0.5),
                             (0.4, 0.3, 0.5))))
    sc1, _, _ = build_config1(ctx, 16, 16)
    out.append(("config 1 (BVH stress)", sc1, N.RT_RENDER_NEE_AREA,
                random_views(rng, int(counts[1]), (-0.6, -0.6, 2.0), (0.6, 0.6, 4.0), (-0.3, -0.3, -0.3),
                             (0.3, 0.3, 0.3))))
    sc2, _, _ = build_config2(ctx, 16, 16)
    out.append(("config 2 (guiding room)", sc2, N.RT_RENDER_NEE_AREA,
                random_views(rng, int(counts[2]), (-1.7, 0.4, -1.7), (1.7, 2.2, 0.8), (-1.9, 0.0, -1.9),
                             (1.9, 1.5, 0.5))))
    return out


# Config 4 photon map and render modes: photons traced per map, the gather size, and the
# render flags — RENDER_MODE HYBRID (at each scattering vertex the direct term is the mean of
# the photon density and point-light NEE, and the path continues, so the guide has bounces to
# sample) with CHECK_SUBSURFACE_SCATTERING (the dipole estimate at camera hits on the slab).
CONFIG4_PHOTONS = 10_000_000
CONFIG4_K = 50
CONFIG4_FLAGS = N.RT_RENDER_HYBRID | N.RT_RENDER_SUBSURFACE


def build_config4(ctx, width=3840, height=2160, seed=11, n=1000):
    """Config 4 scene: terrain (Lambertian 0.6/0.55/0.45, shape 0), the slab (SSMaterial,
    shape 1), 16 glass spheres (shapes 100-115), point lights of 50 RGB at (-1.6, 2.6, 1.4)
    and (1.8, 3.2, -1.2); camera at (0, 2.4, 5.6) looking at (0, -0.1, 0), 45 degrees."""
    (tv, tf), (sv, sf), spheres = scenes.photon_terrain(seed=seed, n=n)
    mats = [core.material(N.RT_MAT_LAMBERTIAN, color=(0.6, 0.55, 0.45)),
            core.material(N.RT_MAT_DIELECTRIC, color=(1, 1, 1), ior=1.5, transparent=True),
            core.subsurface_material(kd=(0.9, 0.9, 0.9), ks=(0.04, 0.04, 0.04), ns=40.0, eta=1.3,
                                     sigma_s=(1.0, 0.8, 0.6), sigma_a=(0.01, 0.02, 0.05), g=0.0)]
    sc = core.Scene(ctx)
    sc.set_materials(mats)
    sc.add_mesh(tv, tf, material=0, shape_id=0)
    sc.add_mesh(sv, sf, material=2, shape_id=1)
    for j, (c, r) in enumerate(spheres):
        o2w, w2o = scenes.sphere_matrices(c, r)
        sc.add_sphere(o2w, w2o, r, material=1, shape_id=100 + j, transparent=True)
    sc.add_point_light((-1.6, 2.6, 1.4), (1.0, 1.0, 1.0), 50.0)
    sc.add_point_light((1.8, 3.2, -1.2), (1.0, 1.0, 1.0), 50.0)
    sc.commit()
    cam = core.look_at_camera((0.0, 2.4, 5.6), (0.0, -0.1, 0.0), (0, 1, 0), 45.0, width, height)
    return sc, cam, dict(spp=256, max_depth=16, rr_depth=3)


# The config-4 guide covers the terrain's bounding box (the slab and spheres lie inside it).
CONFIG4_GUIDE = dict(GUIDE_TRAINING, bbox_min=(-4.01, -0.41, -4.01), bbox_max=(4.01, 1.21, 4.01))
