"""SSMaterial::singleScattering (materials/SSMaterial.cu:108-181) on the GPU
(rt_material_single_scattering) against the reference's own class (oracle/_ref, its host code)
on the same inputs and the same sampler sample: value, refracted light direction and entry
point. The reference keeps spectra in double and scalars in float; the device does the same,
up to the order of a few float products, so the tolerance is relative 1e-4."""
import ctypes
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")


def unit(v):
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32).reshape(-1)).cuda()


@pytest.mark.parametrize("eta,g,ss,sa", [(1.3, 0.0, (1.0, 0.8, 0.6), (0.05, 0.1, 0.2)),
                                         (1.5, 0.4, (2.0, 1.5, 0.9), (0.3, 0.02, 0.1)),
                                         (1.1, -0.3, (0.7, 0.7, 0.7), (0.01, 0.01, 0.5))])
def test_single_scattering_matches_reference(core, gpu_ctx, eta, g, ss, sa):
    import torch
    from oracle import bindings

    try:
        ref = bindings.RefRender()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    rng = np.random.default_rng(int(eta * 100) + int(g * 10))
    n = 2000
    wo = rng.normal(size=(n, 3))
    wo[:, 2] = np.abs(wo[:, 2]) + 0.05
    wo = unit(wo).astype(np.float32)
    L = unit(rng.normal(size=(n, 3)))
    L = L[np.abs(L[:, 2]) > 0.05][: n // 2]  # the entry point is where the light ray meets z = 0
    wo = wo[: L.shape[0]]
    L = L.astype(np.float32)
    L[0] = 0.0  # the photon case: no light direction, value 0
    seeds = np.arange(1, L.shape[0] + 1, dtype=np.uint32) * 7919
    v_ref, wi_ref, pt_ref, u = ref.single_scattering(eta, 20.0, g, ss, sa, wo, L, seeds)
    m = core.subsurface_material((0.5, 0.5, 0.5), (0.1, 0.1, 0.1), 20.0, eta, ss, sa, g=g)
    k = wo.shape[0]
    rgb = torch.zeros(3 * k, dtype=torch.float32, device="cuda")
    wi = torch.zeros(3 * k, dtype=torch.float32, device="cuda")
    pt = torch.zeros(3 * k, dtype=torch.float32, device="cuda")
    # the device inputs stay referenced until the call returns (a temporary's memory could be
    # handed to the next allocation)
    wo_d, L_d, u_d = cuda(wo), cuda(L), cuda(u)
    N.check(N.lib().rt_material_single_scattering(ctypes.byref(m), wo_d.data_ptr(), L_d.data_ptr(), u_d.data_ptr(), k,
                                                  rgb.data_ptr(), wi.data_ptr(), pt.data_ptr()))
    v = rgb.view(k, 3).cpu().numpy()
    w = wi.view(k, 3).cpu().numpy()
    p = pt.view(k, 3).cpu().numpy()
    assert np.all(v[0] == 0) and np.all(v_ref[0] == 0)
    assert np.all(np.isfinite(v_ref[1:])) and np.all(np.isfinite(v[1:]))
    assert np.allclose(v[1:], v_ref[1:], rtol=1e-4, atol=1e-7), np.abs(v - v_ref)[1:].max()
    assert np.allclose(w[1:], wi_ref[1:], rtol=1e-5, atol=1e-5)
    scale = np.maximum(np.abs(pt_ref[1:]).max(axis=1, keepdims=True), 1.0)
    assert np.allclose(p[1:] / scale, pt_ref[1:] / scale, rtol=1e-4, atol=1e-5)


def test_single_scattering_rejects_other_materials(core, gpu_ctx):
    m = core.material(N.RT_MAT_LAMBERTIAN)
    rc = N.lib().rt_material_single_scattering(ctypes.byref(m), None, None, None, 0, None, None, None)
    assert rc != 0
