"""The drop-in layer (include/rt_b200_compat.hpp) maps the reference's BeckmannMaterial,
TrowbridgeBasicMaterial, FresnelBlendMaterial and PlasticUnrealMaterial objects to the core's
material types with the fields the core's BSDFs read (CPU: no GPU call)."""
import ctypes
import importlib

import numpy as np
import pytest

N = importlib.import_module("2023_render_engine_b200._native")


@pytest.fixture(scope="module")
def refc():
    from oracle import bindings

    try:
        return bindings.RefCompat()
    except (FileNotFoundError, OSError) as e:
        pytest.skip(str(e))


def mapped(refc, kind, kd, eta, k, rx, ry):
    arr = [np.asarray(x, np.float32) for x in (kd, eta, k)]
    out = N.Material()
    rc = refc.L.refc_map_material(kind, *[a.ctypes.data for a in arr], rx, ry, ctypes.byref(out))
    assert rc == 0
    return out


@pytest.mark.parametrize("kind,type_", [(1, N.RT_MAT_TROWBRIDGE), (8, N.RT_MAT_BECKMANN), (9, N.RT_MAT_TROWBRIDGE_BASIC)])
def test_microfacet_conductors(refc, kind, type_):
    m = mapped(refc, kind, (0.7, 0.5, 0.3), (0.2, 0.9, 1.1), (3.9, 2.4, 2.2), 0.3, 0.1)
    assert m.type == type_
    assert np.allclose(list(m.color), (0.7, 0.5, 0.3)) and np.allclose(list(m.eta), (0.2, 0.9, 1.1))
    assert np.allclose(list(m.k), (3.9, 2.4, 2.2))
    # the BSDFs keep alpha = sqrt(roughness); the core takes the roughness back
    assert np.allclose(list(m.roughness), (0.3, 0.1), rtol=1e-6)


def test_fresnel_blend_and_plastic(refc):
    fb = mapped(refc, 10, (2.0, 1.0, 0.5), (1, 1, 1), (0, 0, 0), 0, 0)
    assert fb.type == N.RT_MAT_FRESNEL_BLEND and np.allclose(list(fb.extra), (2.0, 1.0, 0.5))  # ke
    pu = mapped(refc, 11, (0.6, 0.5, 0.4), (1, 1, 1), (0, 0, 0), 0, 0)
    assert pu.type == N.RT_MAT_PLASTIC and np.allclose(list(pu.color), (0.6, 0.5, 0.4))


@pytest.mark.parametrize("kind,type_,textured", [
    (0, N.RT_MAT_LAMBERTIAN, True), (1, N.RT_MAT_TROWBRIDGE, True), (3, N.RT_MAT_PLAIN, True),
    (5, N.RT_MAT_PHONG, True), (6, N.RT_MAT_SUBSURFACE, True), (8, N.RT_MAT_BECKMANN, True),
    (9, N.RT_MAT_TROWBRIDGE_BASIC, True), (10, N.RT_MAT_FRESNEL_BLEND, False)])
def test_drop_in_reports_each_material_texture(refc, tmp_path, kind, type_, textured):
    """The layer hands every material's Texture (the member its class reads) to the scene for
    registration; FresnelBlend's texture is never read by the reference, so it is not."""
    from oracle import bindings

    bmp = tmp_path / "tex.bmp"
    bindings.write_bmp24(bmp, np.random.default_rng(kind).integers(0, 256, size=(4, 8, 3), dtype=np.uint8))
    out = N.Material()
    has = ctypes.c_int(-1)
    L = refc.L
    L.refc_map_textured.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p]
    L.refc_map_textured.restype = ctypes.c_int
    assert L.refc_map_textured(kind, str(bmp).encode(), ctypes.byref(out), ctypes.byref(has)) == 0
    assert out.type == type_
    assert has.value == (1 if textured else 0)
    assert out.texture == 0  # the scene sets the id when it registers the texture
