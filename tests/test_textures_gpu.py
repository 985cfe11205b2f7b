"""Textures on the GPU: rt_texture_lookup against the reference's own Texture::getColor
(bit-exact); renders of textured materials against the same renders with the texel folded
into the material by hand (bit-exact: the texture path must do exactly the documented
multiply or replace, in the path tracer, the photon tracer and the photon gathers); and
image-level parity of textured Plane walls with the reference's own integrator."""
import importlib

import numpy as np
import pytest

from oracle import bindings

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
import test_render_ref_parity as P  # noqa: E402  (the parity scene and its tile z-test)
import test_textures as T  # noqa: E402  (the BMP texels and edge coordinates)


def cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32).reshape(-1)).cuda()


@pytest.mark.parametrize("w,h", [(4, 3), (8, 5), (64, 32)])
def test_texture_lookup_matches_reference_texture(core, gpu_ctx, refo, tmp_path, w, h):
    rng = np.random.default_rng(w + h)
    img = T.texture(rng, w, h)
    path = tmp_path / "tex.bmp"
    bindings.write_bmp24(path, img)
    uv = np.concatenate([np.array(T.EDGE_UV, np.float32), rng.uniform(-0.5, 1.5, size=(5000, 2)).astype(np.float32)])
    ref = bindings.ref_texture_lookup(refo, path, uv)
    sc = core.Scene(gpu_ctx)
    tid = sc.add_texture(img.astype(np.float32) / np.float32(255.0))
    mine = sc.texture_lookup(tid, cuda(uv)).cpu().numpy()
    assert np.array_equal(ref.view(np.uint32), mine.view(np.uint32))


def box_scene(core, ctx, wall_material, texture=None, uvs=False):
    """The five Plane walls of the image-parity scene as triangles (texture coordinates = the
    plane's object-space (x, y) when uvs), a point light; the wall facing the camera gets
    wall_material."""
    sc = core.Scene(ctx)
    mats = [core.material(N.RT_MAT_LAMBERTIAN, color=k) for k in P.KD]
    mats[0] = wall_material  # the wall facing the camera (x = 0.5)
    if texture is not None:
        tid = sc.add_texture(texture)
        assert tid == 0
    sc.set_materials(mats)
    v, f = P.plane_triangles()
    for i in range(len(P.PLANES)):
        sc.add_mesh(v, f[2 * i:2 * i + 2], material=i, shape_id=i)
    if uvs:
        quad = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], np.float32)
        sc.set_triangle_uvs(0, np.tile(quad, (len(P.PLANES), 1, 1)))
    sc.add_point_light(*P.LIGHT)
    sc.commit()
    return sc


def camera(w=64, h=64):
    cam = N.Camera()
    # from (-1.75, 0, 0) along +x (camera z), 90 degree field of view
    c2w = np.array([[0, 0, 1, -1.75], [1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1]], np.float32)
    r2c = np.array([[2.0 / w, 0, 0, -1.0], [0, -2.0 / h, 0, 1.0], [0, 0, 0, 1.0], [0, 0, 0, 1]], np.float32)
    cam.camera_to_world[:] = [float(x) for x in c2w.reshape(-1)]
    cam.raster_to_camera[:] = [float(x) for x in r2c.reshape(-1)]
    cam.lens_radius, cam.focal_distance, cam.width, cam.height = 0.0, 0.0, w, h
    return cam


TEXEL = np.array([[[0.9, 0.35, 0.6]]], np.float32)  # a 1x1 texture: every surface point reads it


def kd_eff(type_, color):
    c = np.asarray(color, np.float32)
    if type_ in (N.RT_MAT_LAMBERTIAN, N.RT_MAT_PHONG, N.RT_MAT_SUBSURFACE, N.RT_MAT_PLAIN):
        return c * TEXEL[0, 0]
    if type_ in (N.RT_MAT_TROWBRIDGE, N.RT_MAT_TROWBRIDGE_BASIC, N.RT_MAT_BECKMANN):
        return TEXEL[0, 0].copy()
    return c


MATERIALS = {
    "lambertian": dict(type_=N.RT_MAT_LAMBERTIAN, color=(0.8, 0.7, 0.6)),
    "phong": dict(type_=N.RT_MAT_PHONG, color=(0.5, 0.6, 0.7), k=(0.3, 0.3, 0.3), roughness=(30.0, 0.0)),
    "plain": dict(type_=N.RT_MAT_PLAIN, color=(0.4, 0.8, 0.5)),
    "trowbridge": dict(type_=N.RT_MAT_TROWBRIDGE, color=(0.2, 0.4, 0.9), eta=(0.2, 0.9, 1.1), k=(3.9, 2.4, 2.2),
                       roughness=(0.2, 0.3)),
    "beckmann": dict(type_=N.RT_MAT_BECKMANN, color=(0.6, 0.2, 0.4), eta=(0.2, 0.9, 1.1), k=(3.9, 2.4, 2.2),
                     roughness=(0.2, 0.3)),
    "trowbridge_basic": dict(type_=N.RT_MAT_TROWBRIDGE_BASIC, color=(0.3, 0.3, 0.8), eta=(0.2, 0.9, 1.1),
                             k=(3.9, 2.4, 2.2), roughness=(0.2, 0.3)),
    "fresnel_blend": dict(type_=N.RT_MAT_FRESNEL_BLEND, color=(0.5, 0.5, 0.5)),
    "dielectric": dict(type_=N.RT_MAT_DIELECTRIC, color=(1.0, 1.0, 1.0), ior=1.5),
}


def render(core, sc, flags, seed=11):
    film, _ = sc.render(camera(), spp=4, max_depth=6, rr_depth=3, seed=seed, flags=flags, fp64=True)
    return core.film_mean(film)


@pytest.mark.parametrize("name", sorted(MATERIALS))
def test_textured_material_renders_as_its_folded_kd(core, gpu_ctx, name):
    spec = dict(MATERIALS[name])
    type_ = spec.pop("type_")
    textured = core.material(type_, texture=0, **spec)
    spec["color"] = tuple(float(x) for x in kd_eff(type_, spec["color"]))
    folded = core.material(type_, **spec)
    for flags in (0, N.RT_RENDER_COMPAT):
        a = render(core, box_scene(core, gpu_ctx, textured, texture=TEXEL), flags)
        b = render(core, box_scene(core, gpu_ctx, folded), flags)
        assert np.array_equal(a, b), (name, flags, np.abs(a - b).max())
    if type_ not in (N.RT_MAT_FRESNEL_BLEND, N.RT_MAT_DIELECTRIC):  # the texel must have changed something
        plain = core.material(type_, **{k: v for k, v in MATERIALS[name].items() if k != "type_"})
        c = render(core, box_scene(core, gpu_ctx, plain), N.RT_RENDER_COMPAT)
        assert not np.array_equal(a, c)


def test_textured_photon_trace_and_gathers_use_the_texel(core, gpu_ctx):
    """Hybrid rendering over a photon map: the photon tracer's bounces and the density
    gathers must see the texel exactly as the folded material."""
    imgs = []
    for textured in (True, False):
        kd = (0.8, 0.7, 0.6)
        m = core.material(N.RT_MAT_LAMBERTIAN, color=kd, texture=0 if textured else None)
        if not textured:
            m = core.material(N.RT_MAT_LAMBERTIAN, color=tuple(float(x) for x in kd_eff(N.RT_MAT_LAMBERTIAN, kd)))
        sc = box_scene(core, gpu_ctx, m, texture=TEXEL if textured else None)
        pm, _ = sc.trace_photons(200_000, max_depth=6, seed=3)
        pm.build()
        sc.set_photon_map(pm, k=20, radius=0.2)
        imgs.append(render(core, sc, N.RT_RENDER_HYBRID))
        sc.set_photon_map(None, 20, 0.2)
        pm.close()
    assert np.array_equal(imgs[0], imgs[1]), np.abs(imgs[0] - imgs[1]).max()


def test_textured_planes_match_reference_integrator(core, gpu_ctx, tmp_path):
    """The far wall, the floor and the ceiling carry an 8x4 random texture (Plane surface point = its
    object-space (x, y)); per-tile z-test against the reference's own integrator as in
    test_render_ref_parity."""
    try:
        ref = bindings.RefRender()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    rng = np.random.default_rng(5)
    img = T.texture(rng, 8, 4)
    bmp = tmp_path / "walls.bmp"
    bindings.write_bmp24(bmp, img)
    textured = np.array([1, 0, 0, 1, 1], np.int32)
    path = tmp_path / "box.obejota"
    path.write_text(P.OBEJOTA)
    runs = 8
    R, c2w, r2c = [], None, None
    for _ in range(runs):
        out, c2w, r2c = ref.render(path, P.PLANES, P.KD, bmp_path=bmp, textured=textured)
        R.append(out)
    w, h, spp, depth = ref.width, ref.height, ref.spp, ref.depth
    sc = core.Scene(gpu_ctx)
    tid = sc.add_texture(img.astype(np.float32) / np.float32(255.0))
    sc.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=k, texture=tid if textured[i] else None)
                      for i, k in enumerate(P.KD)])
    v, f = P.plane_triangles()
    for i in range(len(P.PLANES)):
        sc.add_mesh(v, f[2 * i:2 * i + 2], material=i, shape_id=i)
    quad = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], np.float32)
    sc.set_triangle_uvs(0, np.tile(quad, (len(P.PLANES), 1, 1)))
    sc.add_point_light(*P.LIGHT)
    sc.commit()
    cam = N.Camera()
    cam.camera_to_world[:] = [float(x) for x in c2w.reshape(-1)]
    cam.raster_to_camera[:] = [float(x) for x in r2c.reshape(-1)]
    cam.lens_radius, cam.focal_distance, cam.width, cam.height = 0.0, 0.0, w, h
    M = []
    for r in range(runs):
        film, _ = sc.render(cam, spp=spp, max_depth=depth, rr_depth=3, seed=300 + r, flags=N.RT_RENDER_COMPAT,
                            fp64=True)
        M.append(core.film_mean(film))
    Rt = np.stack([P.tiles(i, w, h) for i in R])
    Mt = np.stack([P.tiles(i, w, h) for i in M])
    se = np.sqrt(Rt.var(axis=0, ddof=1) / runs + Mt.var(axis=0, ddof=1) / runs)
    z = (Mt.mean(0) - Rt.mean(0)) / np.maximum(se, 1e-12)
    zs = z[se > 0]
    assert np.abs(zs).mean() < 1.2
    assert (np.abs(zs) > 4).mean() < 0.01
    assert abs(zs.mean()) < 0.25
    assert abs(Mt.mean() - Rt.mean()) / Rt.mean() < 0.01
    # and the texture is visible: without it the image differs well beyond the noise
    sc2 = core.Scene(gpu_ctx)
    sc2.set_materials([core.material(N.RT_MAT_LAMBERTIAN, color=k) for k in P.KD])
    for i in range(len(P.PLANES)):
        sc2.add_mesh(v, f[2 * i:2 * i + 2], material=i, shape_id=i)
    sc2.add_point_light(*P.LIGHT)
    sc2.commit()
    U = np.stack([P.tiles(core.film_mean(sc2.render(cam, spp=spp, max_depth=depth, rr_depth=3, seed=900 + r,
                                                    flags=N.RT_RENDER_COMPAT, fp64=True)[0]), w, h)
                  for r in range(runs)])
    zu = (U.mean(0) - Rt.mean(0)) / np.maximum(np.sqrt(Rt.var(axis=0, ddof=1) / runs + U.var(axis=0, ddof=1) / runs),
                                                1e-12)
    assert (np.abs(zu[se > 0]) > 4).mean() > 0.05


def test_compat_layer_maps_reference_textures(tmp_path):
    """The reference's own Plane + LambertianMaterial(kd, ka, Texture*) objects through the drop-in
    layer (include/rt_b200_compat.hpp registers the Texture and the planes' surface
    coordinates) against the reference's own integrator: per-tile z-test."""
    try:
        ref = bindings.RefRender()
        comp = bindings.RefCompat()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    rng = np.random.default_rng(6)
    bmp = tmp_path / "walls.bmp"
    bindings.write_bmp24(bmp, T.texture(rng, 8, 4))
    textured = np.array([1, 0, 1, 1, 0], np.int32)
    path = tmp_path / "box.obejota"
    path.write_text(P.OBEJOTA)
    runs = 8
    R = np.stack([P.tiles(ref.render(path, P.PLANES, P.KD, bmp_path=bmp, textured=textured)[0], ref.width,
                          ref.height) for _ in range(runs)])
    M = np.stack([P.tiles(comp.render(path, P.PLANES, P.KD, 1700 + r, bmp_path=bmp, textured=textured), comp.width,
                          comp.height) for r in range(runs)])
    se = np.sqrt(R.var(axis=0, ddof=1) / runs + M.var(axis=0, ddof=1) / runs)
    z = (M.mean(0) - R.mean(0)) / np.maximum(se, 1e-12)
    zs = z[se > 0]
    assert np.abs(zs).mean() < 1.2
    assert (np.abs(zs) > 4).mean() < 0.01
    assert abs(zs.mean()) < 0.25
    assert abs(M.mean() - R.mean()) / R.mean() < 0.01
