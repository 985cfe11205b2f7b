"""The renderer's BSDFs (rt_material_eval / rt_material_sample, the code every path vertex
runs) against the reference's own material classes (materials/*.cu, compiled into
oracle/_ref/libref_oracle.so): lightReflected and pdf on random direction pairs; the samplers'
consistency with their densities; renders with each of the compat materials."""
import importlib
import zlib

import numpy as np
import pytest

N = importlib.import_module("2023_render_engine_b200._native")

pytestmark = pytest.mark.gpu


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def directions(rng, n, lower=0.15):
    """Random directions, a fraction of them below the surface; none grazing."""
    w = unit(rng.normal(size=(n, 3)))
    w[:, 2] = np.where(np.abs(w[:, 2]) < 0.02, 0.02 * np.sign(w[:, 2] + 1e-9), w[:, 2])
    w = unit(w)
    flip = rng.uniform(size=n) < lower
    w[:, 2] = np.where(flip, -np.abs(w[:, 2]), np.abs(w[:, 2]))
    return w.astype(np.float32)


KINDS = {
    "lambertian": (N.RT_MAT_LAMBERTIAN, 0),
    "trowbridge": (N.RT_MAT_TROWBRIDGE, 1),
    "beckmann": (N.RT_MAT_BECKMANN, 8),
    "trowbridge_basic": (N.RT_MAT_TROWBRIDGE_BASIC, 9),
    "fresnel_blend": (N.RT_MAT_FRESNEL_BLEND, 10),
    "plastic": (N.RT_MAT_PLASTIC, 11),
}


def make(core, kind, kd, eta, k, rx, ry):
    return core.material(KINDS[kind][0], color=kd, eta=eta, k=k, roughness=(rx, ry))


@pytest.mark.parametrize("kind", list(KINDS))
@pytest.mark.parametrize("rough", [(0.05, 0.05), (0.3, 0.1), (0.8, 0.8)])
def test_eval_matches_reference_classes(core, refo, kind, rough):
    from oracle import bindings

    rng = np.random.default_rng(zlib.crc32(f"{kind}{rough}".encode()))
    n = 4000
    wo, wi = directions(rng, n), directions(rng, n)
    kd, eta, k = (0.7, 0.5, 0.3), (0.2, 0.9, 1.1), (3.9, 2.4, 2.2)
    f, pdf = core.material_eval(make(core, kind, kd, eta, k, *rough), wo, wi)
    rf, rpdf = bindings.ref_material_eval(refo, KINDS[kind][1], kd, eta, k, rough[0], rough[1], wo, wi)
    ok_f = np.isclose(f, rf, rtol=2e-3, atol=1e-6).all(1)
    ok_p = np.isclose(pdf, rpdf, rtol=2e-3, atol=1e-6) | (~np.isfinite(rpdf) & ~np.isfinite(pdf))
    assert ok_f.mean() > 0.999 and ok_p.mean() > 0.999, (kind, np.nonzero(~ok_f)[0][:5], np.nonzero(~ok_p)[0][:5])


def hemisphere_integral(core, mat, wo, m=200_000, seed=0):
    """∫ f|cos| dω over the upper hemisphere by uniform quadrature (f from rt_material_eval)."""
    rng = np.random.default_rng(seed)
    wi = unit(rng.normal(size=(m, 3)))
    wi[:, 2] = np.abs(wi[:, 2])
    f, _ = core.material_eval(mat, np.tile(wo, (m, 1)), wi.astype(np.float32))
    return f.mean(0) * 2 * np.pi


@pytest.mark.parametrize("kind", ["beckmann", "trowbridge_basic", "trowbridge"])
def test_sampler_value_is_f_cos_over_its_density(core, kind):
    """E[sample value] = ∫ f|cos| dω: the value divides by the density the sampler draws from."""
    mat = make(core, kind, (0.8, 0.6, 0.4), (0.2, 0.9, 1.1), (3.9, 2.4, 2.2), 0.3, 0.3)
    wo = unit(np.array([0.4, -0.2, 0.8])).astype(np.float32)
    n = 400_000
    _, val, _, _ = core.material_sample(mat, np.tile(wo, (n, 1)), seed=3)
    est = val.astype(np.float64).mean(0)
    ref = hemisphere_integral(core, mat, wo)
    assert np.allclose(est, ref, rtol=0.03), (est, ref)


def test_plastic_estimator_is_the_references(core):
    """PlasticUnreal: 70% Lambertian (value kd, pdf 0) and 30% mirror (value ks, delta)."""
    mat = make(core, "plastic", (0.6, 0.5, 0.4), (1, 1, 1), (0, 0, 0), 0.0, 0.0)
    wo = np.tile(unit(np.array([0.3, 0.1, 0.9])).astype(np.float32), (100_000, 1))
    wi, val, pdf, delta = core.material_sample(mat, wo, seed=5)
    assert abs(delta.mean() - 0.3) < 0.01
    assert np.allclose(val, (0.6, 0.5, 0.4)) and np.all(pdf == 0)
    assert np.allclose(wi[delta], wo[delta] * np.array([-1, -1, 1]), atol=1e-6)


@pytest.mark.parametrize("kind", ["beckmann", "trowbridge_basic", "fresnel_blend", "plastic"])
@pytest.mark.parametrize("compat", [False, True])
def test_render_with_compat_material(core, gpu_ctx, kind, compat):
    """A floor of the material under a quad emitter: a finite, positive image in both modes."""
    sc = core.Scene(gpu_ctx)
    sc.set_materials([make(core, kind, (0.7, 0.6, 0.5), (0.2, 0.9, 1.1), (3.9, 2.4, 2.2), 0.2, 0.2),
                      core.material(N.RT_MAT_LIGHT, color=(1, 1, 1), intensity=10.0)])
    floor = np.array([[-2, 0, -2], [2, 0, -2], [2, 0, 2], [-2, 0, 2]], np.float32)
    light = np.array([[-0.5, 1.5, -0.5], [-0.5, 1.5, 0.5], [0.5, 1.5, 0.5], [0.5, 1.5, -0.5]], np.float32)
    q = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)
    sc.add_mesh(floor, q, material=0, shape_id=0)
    sc.add_mesh(light, q, material=1, shape_id=1)
    sc.add_point_light((0.5, 1.0, 0.5), (1, 1, 1), 2.0)
    sc.commit()
    cam = core.look_at_camera((0, 1.2, 3.0), (0, 0, 0), (0, 1, 0), 50.0, 48, 32)
    flags = N.RT_RENDER_COMPAT if compat else N.RT_RENDER_NEE_AREA
    film, st = sc.render(cam, spp=16, max_depth=6, seed=1, flags=flags)
    img = core.film_mean(film)
    assert np.all(np.isfinite(img)) and img.mean() > 0
    assert st["extension_rays"] > 0
