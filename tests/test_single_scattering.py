"""SSMaterial::singleScattering (materials/SSMaterial.cu:108-181), restated step by step in
numpy with the device code's precisions (csrc/material_api.cu single_scattering: float scalars,
double spectra), pinned against the reference's own class (oracle/_ref, host code) on the CPU.
The GPU kernel is compared with the reference in tests/test_zzz_single_scattering_gpu.py."""
import numpy as np
import pytest

from oracle import bindings

f32 = np.float32


def length(v):
    return f32(np.sqrt(f32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])))


def normalize(v):
    return (v / length(v)).astype(np.float32)


def refract_ref(d, n, eta_i, eta_t):
    """geometricMath.cu:183-195: the direction scaled by eta_i; total internal reflection: 0."""
    c = f32(np.dot(n, d))
    s2i = max(f32(0), f32(1) - c * c)
    s2t = f32(eta_i * eta_i / (eta_t * eta_t)) * s2i
    if s2t >= 1:
        return np.zeros(3, np.float32)
    ct = f32(np.sqrt(f32(1) - s2t))
    return (d * f32(eta_i) + n * (f32(eta_i) * c - ct)).astype(np.float32)


def fresnel_ref(cos_o, ni, nt):
    """fresnelDielectric as the reference writes it (geometricMath.cu:202-240)."""
    cos_o = f32(min(max(cos_o, -1), 1))
    if not cos_o > 0:
        cos_o = abs(cos_o)
    sin_o = f32(np.sqrt(max(f32(0), f32(1) - cos_o * cos_o)))
    sin_t = f32(ni / nt) * sin_o
    if sin_o >= 1:
        return f32(1)
    cos_t = f32(np.sqrt(max(f32(0), f32(1) - sin_t * sin_t)))
    r = f32((nt * cos_o - nt * cos_t) / (nt * cos_o + nt * cos_t))
    return f32((r * r + r * r) / 2 * abs(cos_o))


def restated(eta, g, sigma_s, sigma_a, wo, L, u):
    """(value, Ti, Pi) of SSMaterial::singleScattering for one case, in the device's steps."""
    if length(L) == 0:
        return np.zeros(3), np.zeros(3), np.zeros(3)
    eta_i, eta_t = f32(1), f32(eta)
    inv_eta = eta_i / eta_t
    sa = np.array(sigma_a, np.float64)
    ss = np.array(sigma_s, np.float64)
    sig_t = sa + ss
    nz = np.array([0, 0, 1], np.float32)
    to = normalize(refract_ref(-wo, nz, eta_i, eta_t))
    sp_o = f32(-np.float64(np.log(f32(u))) / sig_t.max())
    p_o = (to * sp_o).astype(np.float32)
    t = f32(-p_o[2] / L[2])
    pi_ = (p_o + L * t).astype(np.float32)
    si = length(pi_ - p_o)
    lcos = f32(abs(np.dot(L, nz)) / length(L))
    sp_i = f32(si * lcos / np.sqrt(f32(1) - inv_eta * inv_eta * (f32(1) - lcos * lcos)))
    kti = f32(1) - fresnel_ref(f32(np.dot(L, nz) / length(L)), eta_i, eta_t)
    ti = normalize(refract_ref(L, nz, eta_i, eta_t))
    g = f32(g)
    g2 = g * g
    cti = f32(np.dot(ti, to) / (length(ti) * length(to)))
    phase = f32(np.float64(f32(1) - g2) / np.power(np.float64(f32(1) + f32(2) * g * cti + g2), 1.5))
    G = f32(abs(wo[2] / length(wo)) / abs(ti[2] / length(ti)))
    res = np.exp(sig_t * np.float64(-sp_i)) / (sig_t + sig_t * np.float64(G)) * np.float64(phase) * np.float64(kti)
    ss_r = ss * np.float64(f32(1) - g)
    st_r = ss_r + sa
    al = ss_r / st_r
    sig_tr = np.sqrt(sa * 3.0 * st_r)
    zr = np.sqrt((1.0 - al) * 3.0) / sig_tr
    r = length(pi_)
    c1 = zr * (sig_tr + 1.0 / np.sqrt(np.float64(f32(r * r)) + zr * zr))
    ft_o = 1.0 - np.float64(fresnel_ref(f32(wo[2] / length(wo)), f32(1), eta_t))
    ft_i = 1.0 - np.float64(fresnel_ref(f32(ti[2] / length(ti)), f32(1), eta_t))
    return (res * np.float64(np.float32(np.pi)) * c1 * ft_o * ft_i).astype(np.float32), ti, pi_


@pytest.mark.parametrize("eta,g,s_s,s_a", [(1.3, 0.0, (1.0, 0.8, 0.6), (0.05, 0.1, 0.2)),
                                           (1.5, 0.4, (2.0, 1.5, 0.9), (0.3, 0.02, 0.1)),
                                           (1.1, -0.3, (0.7, 0.7, 0.7), (0.01, 0.01, 0.5))])
def test_restated_single_scattering_matches_reference(eta, g, s_s, s_a):
    try:
        ref = bindings.RefRender()
    except (FileNotFoundError, OSError) as e:
        pytest.skip(str(e))
    rng = np.random.default_rng(1)
    n = 1500
    wo = rng.normal(size=(n, 3))
    wo[:, 2] = np.abs(wo[:, 2]) + 0.05
    wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
    L = rng.normal(size=(n, 3))
    L = L / np.linalg.norm(L, axis=1, keepdims=True)
    keep = np.abs(L[:, 2]) > 0.05
    L, wo = L[keep].astype(np.float32), wo[keep]
    L[0] = 0  # the photon case: value 0
    seeds = np.arange(1, L.shape[0] + 1, dtype=np.uint32) * 7919
    v_ref, wi_ref, pt_ref, u = ref.single_scattering(eta, 20.0, g, s_s, s_a, wo, L, seeds)
    for i in range(L.shape[0]):
        v, w, p = restated(eta, g, s_s, s_a, wo[i], L[i], u[i])
        if i == 0:
            assert np.all(v == 0) and np.all(v_ref[0] == 0)
            continue
        assert np.allclose(v, v_ref[i], rtol=1e-4, atol=1e-7), (i, v, v_ref[i])
        assert np.allclose(w, wi_ref[i], rtol=1e-5, atol=1e-5), (i, w, wi_ref[i])
        sc = max(np.abs(pt_ref[i]).max(), 1.0)
        assert np.allclose(p / sc, pt_ref[i] / sc, rtol=1e-4, atol=1e-5), (i, p, pt_ref[i])
