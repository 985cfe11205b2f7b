"""Textures on the CPU, against the reference's own code (oracle/_ref): the texel index rule of
Texture::getColor (textures/Texture.cu:179-192) restated here exactly as the device code
computes it (csrc/surface.cuh tex_index), and the way each material applies the texel (csrc/
surface.cuh texture_bsdf: multiply kd, replace kd, or ignore), checked as
lightReflected(kd, Texture at uv) == lightReflected(kd_eff) of the reference's own classes."""
import ctypes
import importlib

import numpy as np
import pytest

from oracle import bindings

N = importlib.import_module("2023_render_engine_b200._native")


def tex_index(c, size):
    """Texel index along one axis: float product, x86-64 float -> unsigned conversion (through
    a signed 64-bit integer, low 32 bits kept; NaN / out of range: 0), min(size - 1)."""
    x = np.float32(c) * np.float32(size)
    i = int(np.trunc(x)) if abs(float(x)) < 9.22337204e18 else -(1 << 63)
    return min(i & 0xFFFFFFFF, size - 1)


def restated_lookup(rgb_rows, uv):
    h, w, _ = rgb_rows.shape
    return np.array([rgb_rows[tex_index(v, h), tex_index(u, w)] for u, v in uv], np.float32)


def texture(rng, w, h):
    return rng.integers(0, 256, size=(h, w, 3), dtype=np.uint8)


EDGE_UV = [(0, 0), (1, 1), (0.999999, 0.5), (1.0000001, 0.5), (-0.01, 0.3), (-0.99, 0.3), (-1.0, 0.3), (-3.7, 0.2),
           (2.5, -7.25), (1e6, 0.1), (-1e6, 0.1), (1e30, -1e30), (0.25, 0.75)]  # NaN: Point2f asserts


@pytest.mark.parametrize("w,h", [(4, 3), (8, 5), (16, 16)])
def test_texel_index_rule_matches_reference_texture(refo, tmp_path, w, h):
    rng = np.random.default_rng(w * 100 + h)
    img = texture(rng, w, h)
    path = tmp_path / "tex.bmp"
    bindings.write_bmp24(path, img)
    uv = np.concatenate([np.array(EDGE_UV, np.float32), rng.uniform(-0.5, 1.5, size=(400, 2)).astype(np.float32)])
    ref = bindings.ref_texture_lookup(refo, path, uv)
    mine = restated_lookup(img.astype(np.float32) / np.float32(255.0), uv)
    assert np.array_equal(ref.view(np.uint32), mine.view(np.uint32))


def kd_eff(kind, kd, texel):
    """csrc/surface.cuh texture_bsdf: Lambertian and Phong multiply kd by the texel;
    Trowbridge, Beckmann and TrowbridgeBasic replace kd with it."""
    kd = np.asarray(kd, np.float32)
    return kd * texel if kind in (0, 5) else texel


@pytest.mark.parametrize("kind", [0, 1, 5, 8, 9])
def test_texture_application_per_material_matches_reference(refo, tmp_path, kind):
    rng = np.random.default_rng(kind)
    img = texture(rng, 8, 4)
    path = tmp_path / "tex.bmp"
    bindings.write_bmp24(path, img)
    n = 256
    wo = rng.normal(size=(n, 3))
    wo[:, 2] = np.abs(wo[:, 2]) + 0.05
    wi = rng.normal(size=(n, 3))
    wi[:, 2] = np.abs(wi[:, 2]) + 0.05
    wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
    wi = (wi / np.linalg.norm(wi, axis=1, keepdims=True)).astype(np.float32)
    uv = rng.uniform(0, 1, size=(n, 2)).astype(np.float32)
    kd, eta, k = (0.7, 0.5, 0.3), (0.2, 0.9, 1.1), (3.9, 2.4, 2.2)
    rx, ry = (20.0, 0.0) if kind == 5 else (0.3, 0.1)
    f_tex, pdf_tex = bindings.ref_material_eval_tex(refo, kind, kd, eta, k, rx, ry, path, uv, wo, wi)
    texels = restated_lookup(img.astype(np.float32) / np.float32(255.0), uv)
    for i in range(0, n, 37):
        kde = kd_eff(kind, kd, texels[i])
        if kind == 5:
            f, pdf = bindings.ref_phong_eval(refo, kde, eta, rx, wo[i:i + 1], wi[i:i + 1])
        else:
            f, pdf = bindings.ref_material_eval(refo, kind, kde, eta, k, rx, ry, wo[i:i + 1], wi[i:i + 1])
        # the reference multiplies in its own order (kd / pi * texel); the restated kd_eff
        # multiplies first: equal to a few ulp
        assert np.allclose(f[0], f_tex[i], rtol=2e-6, atol=1e-12), (i, f[0], f_tex[i])
        assert np.allclose(pdf[0], pdf_tex[i], rtol=1e-6)


def test_material_struct_carries_texture_field():
    m = N.Material()
    assert m.texture == 0  # zero-initialised: no texture
    assert N.Material.texture.offset == 72 and ctypes.sizeof(N.Material) == 76  # as rt_b200.h lays it out
