"""Image-level parity with the reference's OWN integrator (PathTracerIntegrator::render,
compiled from its sources into oracle/_ref/libref_render.so) at equal samples per pixel:
a box of five Plane walls lit by a point light (the arrangement of the reference's
cornellBoxGuion main), rendered by both in the reference-compatible estimator mode, compared
per 4x4-pixel tile with a z-test whose variance comes from independent runs of each side."""
import importlib
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")

PLANES = np.array([  # Plane(bottom-left corner, axisX, axisY, normal), unit squares
    [0.5, -0.5, -0.5, 0, 1, 0, 0, 0, 1, -0.5, 0, 0],
    [0.5, 0.5, -0.5, -1, 0, 0, 0, 0, 1, 0, -0.5, 0],
    [0.5, -0.5, -0.5, -1, 0, 0, 0, 0, 1, 0, 0.5, 0],
    [-0.5, -0.5, -0.5, 1, 0, 0, 0, 1, 0, 0, 0, 0.5],
    [-0.5, -0.5, 0.5, 1, 0, 0, 0, 1, 0, 0, 0, -0.5]], np.float32)
KD = np.array([[1, 1, 1], [0, 1, 0], [1, 0, 0], [0.8, 0.8, 0.8], [1, 1, 1]], np.float32)
LIGHT = ((0.0, 0.0, 0.25), (1.0, 1.0, 1.0), 5.0)
OBEJOTA = textwrap.dedent("""\
    camera
    p -1.75 0 0
    lookat 0 0 0
    up 0 0 1
    cts 0 0 -0.8
    frameY 0.6

    lightPoint l1
    p 0 0 0.25
    c 1 1 1
    i 5
    """)


def plane_triangles():
    v, f = [], []
    for i, p in enumerate(PLANES):
        o, ax, ay = p[0:3], p[3:6], p[6:9]
        v += [o, o + ax, o + ax + ay, o + ay]
        f += [[4 * i, 4 * i + 1, 4 * i + 2], [4 * i, 4 * i + 2, 4 * i + 3]]
    return np.array(v, np.float32), np.array(f, np.uint32)


def tiles(img, w, h, t=4):
    return img.reshape(h // t, t, w // t, t, 3).mean(axis=(1, 3)).reshape(-1, 3)


def test_statistical_parity_with_reference_integrator(core, gpu_ctx, tmp_path):
    from oracle import bindings

    try:
        ref = bindings.RefRender()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    path = tmp_path / "box.obejota"
    path.write_text(OBEJOTA)
    runs = 8
    ref_imgs = []
    for _ in range(runs):
        img, c2w, r2c = ref.render(path, PLANES, KD)
        ref_imgs.append(img)
    w, h, spp, depth = ref.width, ref.height, ref.spp, ref.depth
    sc = core.Scene(gpu_ctx)
    sc.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=k) for k in KD])
    v, f = plane_triangles()
    for i in range(len(PLANES)):
        sc.add_mesh(v, f[2 * i:2 * i + 2], material=i, shape_id=i)
    sc.add_point_light(*LIGHT)
    sc.commit()
    cam = N.Camera()
    cam.camera_to_world[:] = [float(x) for x in c2w.reshape(-1)]
    cam.raster_to_camera[:] = [float(x) for x in r2c.reshape(-1)]
    cam.lens_radius, cam.focal_distance, cam.width, cam.height = 0.0, 0.0, w, h
    my_imgs = []
    for r in range(runs):
        film, _ = sc.render(cam, spp=spp, max_depth=depth, rr_depth=3, seed=100 + r, flags=N.RT_RENDER_COMPAT,
                            fp64=True)
        my_imgs.append(core.film_mean(film))
    R = np.stack([tiles(i, w, h) for i in ref_imgs])   # runs x tiles x 3
    M = np.stack([tiles(i, w, h) for i in my_imgs])
    se = np.sqrt(R.var(axis=0, ddof=1) / runs + M.var(axis=0, ddof=1) / runs)
    z = (M.mean(0) - R.mean(0)) / np.maximum(se, 1e-12)
    valid = se > 0
    zs = z[valid]
    assert np.abs(zs).mean() < 1.2                      # ~0.8 expected under equal means
    assert (np.abs(zs) > 4).mean() < 0.01
    assert abs(zs.mean()) < 0.25
    rel = abs(M.mean() - R.mean()) / R.mean()
    assert rel < 0.01


def test_analytic_planes_match_the_reference_integrator(core, gpu_ctx, refo, tmp_path):
    """The same box with its walls as analytic planes (rt_scene_add_plane with the reference's
    own Plane matrices and Plane::intersects arithmetic) instead of triangles: the per-tile
    z-test against the reference integrator as above."""
    from oracle import bindings

    try:
        ref = bindings.RefRender()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    path = tmp_path / "box.obejota"
    path.write_text(OBEJOTA)
    runs = 8
    ref_imgs = []
    for _ in range(runs):
        img, c2w, r2c = ref.render(path, PLANES, KD)
        ref_imgs.append(img)
    w, h, spp, depth = ref.width, ref.height, ref.spp, ref.depth
    rp = bindings.RefPlanes(refo, PLANES)
    sc = core.Scene(gpu_ctx)
    sc.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=k) for k in KD])
    for i in range(len(PLANES)):
        o2w, w2o = rp.matrices(i)
        sc.add_plane(o2w, w2o, material=i, shape_id=i)
    sc.add_point_light(*LIGHT)
    sc.commit()
    cam = N.Camera()
    cam.camera_to_world[:] = [float(x) for x in c2w.reshape(-1)]
    cam.raster_to_camera[:] = [float(x) for x in r2c.reshape(-1)]
    cam.lens_radius, cam.focal_distance, cam.width, cam.height = 0.0, 0.0, w, h
    my_imgs = []
    for r in range(runs):
        film, _ = sc.render(cam, spp=spp, max_depth=depth, rr_depth=3, seed=900 + r, flags=N.RT_RENDER_COMPAT,
                            fp64=True)
        my_imgs.append(core.film_mean(film))
    R = np.stack([tiles(i, w, h) for i in ref_imgs])
    M = np.stack([tiles(i, w, h) for i in my_imgs])
    se = np.sqrt(R.var(axis=0, ddof=1) / runs + M.var(axis=0, ddof=1) / runs)
    z = (M.mean(0) - R.mean(0)) / np.maximum(se, 1e-12)
    zs = z[se > 0]
    assert np.abs(zs).mean() < 1.2
    assert (np.abs(zs) > 4).mean() < 0.01
    assert abs(zs.mean()) < 0.25
    assert abs(M.mean() - R.mean()) / R.mean() < 0.01


def test_compat_layer_is_a_drop_in_for_the_reference_integrator(tmp_path):
    """The same reference objects (its Plane, LambertianMaterial, loadObejota camera, film and
    point light) through include/rt_b200_compat.hpp — rtb::Scene::build and
    rtb::PathTracerIntegrator::render in place of the reference's — give the reference
    integrator's image (per-tile z-test as above), written into the reference's own Film."""
    from oracle import bindings

    try:
        ref = bindings.RefRender()
        comp = bindings.RefCompat()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    path = tmp_path / "box.obejota"
    path.write_text(OBEJOTA)
    runs = 8
    R = np.stack([tiles(ref.render(path, PLANES, KD)[0], ref.width, ref.height) for _ in range(runs)])
    M = np.stack([tiles(comp.render(path, PLANES, KD, 700 + r), comp.width, comp.height) for r in range(runs)])
    assert (comp.width, comp.height, comp.spp, comp.depth) == (ref.width, ref.height, ref.spp, ref.depth)
    se = np.sqrt(R.var(axis=0, ddof=1) / runs + M.var(axis=0, ddof=1) / runs)
    z = (M.mean(0) - R.mean(0)) / np.maximum(se, 1e-12)
    zs = z[se > 0]
    assert np.abs(zs).mean() < 1.2
    assert (np.abs(zs) > 4).mean() < 0.01
    assert abs(zs.mean()) < 0.25
    assert abs(M.mean() - R.mean()) / R.mean() < 0.01
