// Evaluation and sampling of a material's BSDF on the device for given directions in the
// shading frame (normal +z): the code the renderer runs at every path vertex, exposed for
// tools that tabulate or check a material (Material::lightReflected / pdf / sampleDirection,
// materials/*.cu).
#include "rt_internal.h"
#include "surface.cuh"
#include "tonemap.cuh"

namespace rtb {
namespace {

constexpr int kMB = 128;

// refract as the reference writes it (geometricMath.cu:183-195): the direction is scaled by
// etaI, not by etaI / etaT, and total internal reflection returns the zero vector
__device__ __forceinline__ V3 refract_ref(V3 d, V3 n, float etaI, float etaT)
{
    const float c = dot(n, d);
    const float s2i = fmaxf(0.f, 1.f - c * c);
    const float s2t = etaI * etaI / (etaT * etaT) * s2i;
    if (s2t >= 1.f) return v3(0.f, 0.f, 0.f);
    const float ct = sqrtf(1.f - s2t);
    return d * etaI + n * (etaI * c - ct);
}

__device__ __forceinline__ D3 d3_sqrt(D3 a) { return D3{__dsqrt_rn(a.r), __dsqrt_rn(a.g), __dsqrt_rn(a.b)}; }
__device__ __forceinline__ D3 d3_exp(D3 a) { return D3{exp(a.r), exp(a.g), exp(a.b)}; }

// SSMaterial::singleScattering (materials/SSMaterial.cu:108-181) in the shading frame (normal
// +z) of an RT_MAT_SUBSURFACE material: wo toward the camera, L the light direction, u the
// sampler's one sample. The refracted camera direction To, a depth -log(u) / max(sigma_t)
// along it, the point Pi where the ray from there along L meets the surface, the attenuation
// exp(-sp_i sigma_t) / (sigma_t (1 + G)) with the Henyey-Greenstein phase and the entering
// Fresnel transmission, times pi C1 Ft_o Ft_i of the dipole (sigma_s' = (1 - g) sigma_s). Its
// spectra are double as the reference's Spectrum; scalar steps are float as its Float.
// Returns the value; *wi = Ti (the refracted light direction), *p = Pi.
__device__ D3 single_scattering(const rt_material &m, V3 wo, V3 L, float u, V3 &wi, V3 &p)
{
    wi = v3(0.f, 0.f, 0.f);
    p = v3(0.f, 0.f, 0.f);
    if (length(L) == 0.f) return d3(0.0);  // photon scattering: no light direction
    const float etaI = 1.f, etaT = m.ior, invEta = etaI / etaT;
    const D3 sa{(double)m.extra[0], (double)m.extra[1], (double)m.extra[2]};
    const D3 ss{(double)m.eta[0], (double)m.eta[1], (double)m.eta[2]};
    const float g = m.roughness[1];
    const D3 sig_t = sa + ss;
    const V3 nz = v3(0.f, 0.f, 1.f);
    const V3 To = normalize(refract_ref(-wo, nz, etaI, etaT));
    if (To.x == 0.f && To.y == 0.f && To.z == 0.f) return d3(0.0);
    const double mx = fmax(sig_t.r, fmax(sig_t.g, sig_t.b));
    const float sp_o = (float)(-(double)logf(u) / mx);
    const V3 p_o = To * sp_o;
    const float t = -p_o.z / L.z;
    const V3 Pi = p_o + L * t;
    p = Pi;
    const float si = length(Pi - p_o);
    const float Lcos = fabsf(dot(L, nz)) / length(L);
    const float sp_i = si * Lcos / sqrtf(1.f - invEta * invEta * (1.f - Lcos * Lcos));
    const float Kti = 1.f - fresnel_dielectric_ref(dot(L, nz) / length(L), etaI, etaT);
    const V3 Ti = normalize(refract_ref(L, nz, etaI, etaT));
    const float g2 = g * g;
    const float cti = dot(Ti, To) / (length(Ti) * length(To));
    const float phase = (float)((double)(1.f - g2) / pow((double)(1.f + 2.f * g * cti + g2), 1.5));
    wi = Ti;
    const float G = fabsf(wo.z / length(wo)) / fabsf(Ti.z / length(Ti));
    const D3 sig_tc = sig_t + sig_t * (double)G;
    const D3 res = d3_exp(sig_t * (double)(-sp_i)) / sig_tc * (double)phase * (double)Kti;
    const D3 ss_r = ss * (double)(1.f - g);
    const D3 st_r = ss_r + sa;
    const D3 al = ss_r / st_r;
    const D3 sig_tr = d3_sqrt(sa * 3.0 * st_r);
    const D3 zr = d3_sqrt((d3(1.0) - al) * 3.0) / sig_tr;
    const float r = length(Pi);
    const D3 dist_r = d3_sqrt(d3((double)(r * r)) + zr * zr);
    const D3 C1 = zr * (sig_tr + d3(1.0) / dist_r);
    const double ft_o = 1.0 - (double)fresnel_dielectric_ref(wo.z / length(wo), 1.f, etaT);
    const double ft_i = 1.0 - (double)fresnel_dielectric_ref(Ti.z / length(Ti), 1.f, etaT);
    return res * (double)kPi * C1 * ft_o * ft_i;
}

__global__ void k_single_scattering(rt_material m, const float *__restrict__ wo, const float *__restrict__ L,
                                    const float *__restrict__ u, uint64_t n, float *__restrict__ rgb,
                                    float *__restrict__ wi, float *__restrict__ pt)
{
    const uint64_t i = blockIdx.x * (uint64_t)kMB + threadIdx.x;
    if (i >= n) return;
    V3 w, p;
    const D3 v = single_scattering(m, v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]),
                                   v3(L[3 * i], L[3 * i + 1], L[3 * i + 2]), u[i], w, p);
    rgb[3 * i] = (float)v.r;
    rgb[3 * i + 1] = (float)v.g;
    rgb[3 * i + 2] = (float)v.b;
    if (wi) {
        wi[3 * i] = w.x;
        wi[3 * i + 1] = w.y;
        wi[3 * i + 2] = w.z;
    }
    if (pt) {
        pt[3 * i] = p.x;
        pt[3 * i + 1] = p.y;
        pt[3 * i + 2] = p.z;
    }
}

__global__ void k_material_eval(rt_material m, const float *__restrict__ wo, const float *__restrict__ wi, uint64_t n,
                                float *__restrict__ f, float *__restrict__ pdf)
{
    const uint64_t i = blockIdx.x * (uint64_t)kMB + threadIdx.x;
    if (i >= n) return;
    const Bsdf b = load_bsdf(m);
    float p = 0.f;
    const V3 v = bsdf_eval(b, v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), p);
    f[3 * i] = v.x;
    f[3 * i + 1] = v.y;
    f[3 * i + 2] = v.z;
    if (pdf) pdf[i] = p;
}

__global__ void k_material_sample(rt_material m, const float *__restrict__ wo, uint64_t n, uint32_t seed, int compat,
                                  float *__restrict__ wi, float *__restrict__ value, float *__restrict__ pdf,
                                  uint8_t *__restrict__ delta)
{
    const uint64_t i = blockIdx.x * (uint64_t)kMB + threadIdx.x;
    if (i >= n) return;
    const Bsdf b = load_bsdf(m);
    Pcg r = pcg_init((uint32_t)i, (uint32_t)(i >> 32), seed);
    V3 w;
    float p = 0.f;
    bool d = false;
    const V3 v = bsdf_sample(b, v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), r, compat != 0, w, p, d);
    wi[3 * i] = w.x;
    wi[3 * i + 1] = w.y;
    wi[3 * i + 2] = w.z;
    value[3 * i] = v.x;
    value[3 * i + 1] = v.y;
    value[3 * i + 2] = v.z;
    if (pdf) pdf[i] = p;
    if (delta) delta[i] = d ? 1 : 0;
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

int rt_material_eval(const rt_material *m, const float *wo, const float *wi, uint64_t n, float *f, float *pdf)
{
    if (!m || (n && (!wo || !wi || !f))) return fail(RT_ERR_INVALID, "rt_material_eval: null argument");
    if (n == 0) return RT_OK;
    k_material_eval<<<(unsigned)((n + kMB - 1) / kMB), kMB>>>(*m, wo, wi, n, f, pdf);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaDeviceSynchronize());
    return RT_OK;
}

int rt_material_sample(const rt_material *m, const float *wo, uint64_t n, uint32_t seed, uint32_t flags, float *wi,
                       float *value, float *pdf, uint8_t *delta)
{
    if (!m || (n && (!wo || !wi || !value))) return fail(RT_ERR_INVALID, "rt_material_sample: null argument");
    if (n == 0) return RT_OK;
    k_material_sample<<<(unsigned)((n + kMB - 1) / kMB), kMB>>>(*m, wo, n, seed, (flags & RT_RENDER_COMPAT) ? 1 : 0, wi,
                                                               value, pdf, delta);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaDeviceSynchronize());
    return RT_OK;
}

int rt_material_single_scattering(const rt_material *m, const float *wo, const float *L, const float *u, uint64_t n,
                                  float *rgb, float *wi, float *point)
{
    if (!m || (n && (!wo || !L || !u || !rgb))) return fail(RT_ERR_INVALID, "rt_material_single_scattering: null argument");
    if (m->type != RT_MAT_SUBSURFACE)
        return fail(RT_ERR_INVALID, "rt_material_single_scattering: not an RT_MAT_SUBSURFACE material");
    if (n == 0) return RT_OK;
    k_single_scattering<<<(unsigned)((n + kMB - 1) / kMB), kMB>>>(*m, wo, L, u, n, rgb, wi, point);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaDeviceSynchronize());
    return RT_OK;
}

}  // extern "C"
