// Device-side shading: RNG, sampling warps, BSDFs and the reference estimator's pieces.
// Each function cites the reference code whose behaviour it reproduces
// (hsunekichi/2023_render_engine).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rt_internal.h"

namespace rtb {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;

// ------------------------------------------------------------------ vectors

struct V3 {
    float x, y, z;
};
__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator*(float s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / length(a)); }
__host__ __device__ __forceinline__ V3 vabs(V3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__host__ __device__ __forceinline__ bool is_black(V3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
// Spectrum::brightness (radiometry/Spectrum.cu:67-75)
__host__ __device__ __forceinline__ float luminance(V3 a) { return 0.212671f * a.x + 0.715160f * a.y + 0.072169f * a.z; }

// ---------------------------------------------------------------------- RNG

// PCG32 (O'Neill): one stream per (pixel, sample): state seeded from the pixel index,
// increment from the sample index and the render seed.
struct Pcg {
    uint64_t state, inc;
};
__host__ __device__ __forceinline__ uint32_t pcg_next(Pcg &r)
{
    uint64_t old = r.state;
    r.state = old * 6364136223846793005ull + r.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
__host__ __device__ __forceinline__ Pcg pcg_init(uint32_t pixel, uint32_t sample, uint32_t seed)
{
    Pcg r;
    r.state = 0u;
    r.inc = ((((uint64_t)sample << 32) | seed) << 1u) | 1u;
    pcg_next(r);
    r.state += (uint64_t)pixel;
    pcg_next(r);
    return r;
}
// uniform in [0, 1)
__host__ __device__ __forceinline__ float pcg_float(Pcg &r) { return (float)(pcg_next(r) >> 8) * (1.0f / 16777216.0f); }

// ------------------------------------------------------------------- warps

// Sampling::concentricSampleDisk (sampling/Sampler.cu:12-36)
__device__ __forceinline__ void concentric_disk(float u1, float u2, float &dx, float &dy)
{
    float ox = 2.0f * u1 - 1.0f, oy = 2.0f * u2 - 1.0f;
    if (ox == 0.f && oy == 0.f) {
        dx = dy = 0.f;
        return;
    }
    float r, th;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        th = (kPi / 4) * (oy / ox);
    } else {
        r = oy;
        th = (kPi / 2) - (kPi / 4) * (ox / oy);
    }
    float s, c;
    sincosf(th, &s, &c);
    dx = r * c;
    dy = r * s;
}

// Sampling::cosineSampleHemisphere (Sampler.cu:73-90)
__device__ __forceinline__ V3 cosine_hemisphere(float u1, float u2)
{
    float x, y;
    concentric_disk(u1, u2, x, y);
    return v3(x, y, sqrtf(fmaxf(0.f, 1.f - x * x - y * y)));
}

// Sampling::uniformSampleSphere (Sampler.cu:46-52)
__device__ __forceinline__ V3 uniform_sphere(float u1, float u2)
{
    float phi = 2 * kPi * u1;
    float cth = 2 * u2 - 1;
    float sth = sqrtf(fmaxf(0.f, 1 - cth * cth));
    float s, c;
    sincosf(phi, &s, &c);
    return v3(sth * c, sth * s, cth);
}

// ------------------------------------------------------------------ Fresnel

// fresnelDielectric exactly as the reference writes it (cuda_libraries/geometricMath.cu:202-240):
// the exit branch swaps an index with itself, both polarisations use the same formula and the
// final expression is (r_par^2 + r_perp^2) / 2 * |cos|.
__device__ __forceinline__ float fresnel_dielectric_ref(float cosO, float ni, float nt)
{
    cosO = fminf(fmaxf(cosO, -1.f), 1.f);
    if (!(cosO > 0)) cosO = fabsf(cosO);
    float sinO = sqrtf(fmaxf(0.f, 1 - cosO * cosO));
    float sinT = ni / nt * sinO;
    if (sinO >= 1) return 1.f;
    float cosT = sqrtf(fmaxf(0.f, 1 - sinT * sinT));
    float r = ((nt * cosO) - (nt * cosT)) / ((nt * cosO) + (nt * cosT));
    return (r * r + r * r) / 2 * fabsf(cosO);
}

// Unpolarised dielectric Fresnel reflectance (physically consistent mode).
__device__ __forceinline__ float fresnel_dielectric(float cosI, float etaI, float etaT)
{
    cosI = fminf(fmaxf(cosI, -1.f), 1.f);
    if (cosI < 0) {
        float t = etaI;
        etaI = etaT;
        etaT = t;
        cosI = -cosI;
    }
    float sinI = sqrtf(fmaxf(0.f, 1 - cosI * cosI));
    float sinT = etaI / etaT * sinI;
    if (sinT >= 1) return 1.f;
    float cosT = sqrtf(fmaxf(0.f, 1 - sinT * sinT));
    float rpar = ((etaT * cosI) - (etaI * cosT)) / ((etaT * cosI) + (etaI * cosT));
    float rper = ((etaI * cosI) - (etaT * cosT)) / ((etaI * cosI) + (etaT * cosT));
    return 0.5f * (rpar * rpar + rper * rper);
}

struct Cx {
    float re, im;
};
__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx csub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx cdiv(Cx a, Cx b)
{
    float s = 1.0f / (b.re * b.re + b.im * b.im);
    return {s * (a.re * b.re + a.im * b.im), s * (a.im * b.re - a.re * b.im)};
}
__device__ __forceinline__ float cnorm(Cx a) { return a.re * a.re + a.im * a.im; }
__device__ __forceinline__ Cx csqrt(Cx z)
{
    // principal root
    float m = sqrtf(cnorm(z));
    float re = sqrtf(fmaxf(0.f, 0.5f * (m + z.re)));
    float im = sqrtf(fmaxf(0.f, 0.5f * (m - z.re)));
    return {re, z.im < 0 ? -im : im};
}

// fresnelConductor(cos, eta + i k) (geometricMath.cu:242-261)
__device__ __forceinline__ float fresnel_conductor(float cosI, float eta, float k)
{
    cosI = fminf(fmaxf(cosI, 0.f), 1.f);
    float sin2 = 1 - cosI * cosI;
    Cx e = {eta, k};
    Cx sin2T = cdiv(Cx{sin2, 0.f}, cmul(e, e));
    Cx cosT = csqrt(csub(Cx{1.f, 0.f}, sin2T));
    Cx ec = cmul(e, Cx{cosI, 0.f});
    Cx rpar = cdiv(csub(ec, cosT), cadd(ec, cosT));
    Cx ect = cmul(e, cosT);
    Cx rper = cdiv(csub(Cx{cosI, 0.f}, ect), cadd(Cx{cosI, 0.f}, ect));
    return (cnorm(rpar) + cnorm(rper)) / 2;
}

// ----------------------------------------------------- Trowbridge-Reitz (GGX)

// TrowbridgeBSDF (materials/TrowbridgeBSDF.cu:12-253), shading space (z = normal).
struct Ggx {
    float ax, ay;
};
__device__ __forceinline__ float cos2t(V3 w) { return w.z * w.z; }
__device__ __forceinline__ float sin2t(V3 w) { return fmaxf(0.f, 1 - cos2t(w)); }
__device__ __forceinline__ float tan2t(V3 w) { return sin2t(w) / cos2t(w); }
__device__ __forceinline__ float cosphi(V3 w)
{
    float s = sqrtf(sin2t(w));
    return s == 0 ? 1.f : fminf(fmaxf(w.x / s, -1.f), 1.f);
}
__device__ __forceinline__ float sinphi(V3 w)
{
    float s = sqrtf(sin2t(w));
    return s == 0 ? 0.f : fminf(fmaxf(w.y / s, -1.f), 1.f);
}
__device__ __forceinline__ float ggx_D(const Ggx &g, V3 h)
{
    float t2 = tan2t(h);
    if (isinf(t2)) return 0.f;
    float c4 = cos2t(h) * cos2t(h);
    float cp = cosphi(h) / g.ax, sp = sinphi(h) / g.ay;
    float e = t2 * (cp * cp + sp * sp);
    return 1.0f / (kPi * g.ax * g.ay * c4 * (1 + e) * (1 + e));
}
__device__ __forceinline__ float ggx_lambda(const Ggx &g, V3 w)
{
    float t2 = tan2t(w);
    if (isinf(t2)) return 0.f;
    float cp = cosphi(w) * g.ax, sp = sinphi(w) * g.ay;
    float a2 = cp * cp + sp * sp;
    return (sqrtf(1 + a2 * t2) - 1) / 2;
}
__device__ __forceinline__ float abs_cos(V3 w) { return fabsf(w.z / length(w)); }
__device__ __forceinline__ float abs_cos2(V3 a, V3 b) { return fabsf(dot(a, b)) / (length(a) * length(b)); }

// visible-normal pdf: G1(wo)/|cos wo| * D(h) * |cos(wo, h)|
__device__ __forceinline__ float ggx_pdf_h(const Ggx &g, V3 wo, V3 h)
{
    return (1.0f / (1 + ggx_lambda(g, wo))) / abs_cos(wo) * ggx_D(g, h) * abs_cos2(wo, h);
}

// lightReflected: D F G / (4 cos_i cos_o) * kd * |cos_i| (F = 1 for TrowbridgeBasicBSDF,
// TrowbridgeBasicBSDF.cu:185-186)
__device__ __forceinline__ V3 ggx_eval(const Ggx &g, V3 kd, V3 eta, V3 k, V3 wo, V3 wi, bool unit_fresnel = false)
{
    wo = normalize(wo);
    wi = normalize(wi);
    if (!(wo.z * wi.z > 0)) return v3(0, 0, 0);
    if (fmaxf(g.ax, g.ay) < 1e-3f) return v3(0, 0, 0);
    float co = abs_cos(wo), ci = abs_cos(wi);
    if (ci == 0 || co == 0) return v3(0, 0, 0);
    V3 h = wi + wo;
    if (dot(h, h) == 0) return v3(0, 0, 0);
    h = normalize(h);
    float c = abs_cos2(wo, h);
    V3 F = unit_fresnel ? v3(1, 1, 1)
                        : v3(fresnel_conductor(c, eta.x, k.x), fresnel_conductor(c, eta.y, k.y),
                             fresnel_conductor(c, eta.z, k.z));
    float D = ggx_D(g, h);
    float G = 1.0f / (1 + ggx_lambda(g, wo) + ggx_lambda(g, wi));
    return F * (D * G / (4 * ci * co)) * kd * ci;
}

__device__ __forceinline__ float ggx_pdf(const Ggx &g, V3 wo, V3 wi)
{
    if (!(wo.z * wi.z > 0)) return 0.f;
    if (fmaxf(g.ax, g.ay) < 1e-3f) return 0.f;
    V3 h = wo + wi;
    if (dot(h, h) == 0) return 0.f;
    h = normalize(h);
    if (h.z < 0) h = -h;  // faceForward(h, +z)
    return ggx_pdf_h(g, wo, h) / (4 * abs_cos2(wo, h));
}

// sampleHalf (TrowbridgeBSDF.cu:120-151): visible normals of the stretched hemisphere.
__device__ __forceinline__ V3 ggx_sample_h(const Ggx &g, V3 wo, float u1, float u2)
{
    V3 wh = normalize(v3(g.ax * wo.x, g.ay * wo.y, wo.z));
    if (wh.z < 0) wh = -wh;
    V3 T1 = (wh.z < 0.99999f) ? normalize(cross(v3(0, 0, 1), wh)) : v3(1, 0, 0);
    V3 T2 = cross(wh, T1);
    // uniformSampleDisk of (2u - 1) (Sampler.cu:38-44)
    float sx = 2 * u1 - 1, sy = 2 * u2 - 1;
    float r = sqrtf(fabsf(sx)), th = 2 * kPi * sy;
    float s, c;
    sincosf(th, &s, &c);
    float px = r * c, py = r * s;
    float hh = sqrtf(1 - px * px);
    float t = (1 + wh.z) / 2;
    py = (1 - t) * hh + t * py;
    float pz = sqrtf(fmaxf(0.f, 1 - (px * px + py * py)));
    V3 nh = T1 * px + T2 * py + wh * pz;
    return normalize(v3(g.ax * nh.x, g.ay * nh.y, fmaxf(1e-6f, nh.z)));
}

// Beckmann distribution and Smith lambda (geometricMath.cu:377-421) of a direction as given:
// the reference also evaluates D at unnormalised sums of directions (BeckmannBSDF::pdf,
// FresnelBlendMaterial::pdf), where cos2t is h.z^2 of the raw vector.
__device__ __forceinline__ float beckmann_D(V3 h, float ax, float ay)
{
    const float t2 = tan2t(h);
    if (isinf(t2)) return 0.f;
    const float c4 = cos2t(h) * cos2t(h);
    const float denom = kPi * ax * ay * c4;
    const float cp = cosphi(h), sp = sinphi(h);
    const float p = fabsf(cp * cp) / (ax * ax) + fabsf(sp * sp) / (ay * ay);
    return expf(-t2 * p) / denom;
}
__device__ __forceinline__ float beckmann_lambda(V3 w, float ax, float ay)
{
    const float tt = fabsf(sqrtf(sin2t(w)) / (w.z / length(w)));
    if (isinf(tt)) return 0.f;
    const float cp = cosphi(w), sp = sinphi(w);
    const float alpha = sqrtf(fabsf(cp * cp) * ax * ax + fabsf(sp * sp) * ay * ay);
    const double a = 1.0 / (alpha * tt);
    if (a >= 1.6) return 0.f;
    return (float)((1 - 1.259 * a + 0.396 * a * a) / (3.535 * a + 2.181 * a * a));
}
// sampleHalfBeckman (BeckmannBSDF.cu:89-110): tan^2 = -ax ay log(1 - u1), phi = 2 pi u2, on
// wo's side
__device__ __forceinline__ V3 beckmann_sample_h(V3 wo, float ax, float ay, float u1, float u2)
{
    float lg = logf(1 - u1);
    if (isinf(lg)) lg = 0.f;
    const float t2 = -ax * ay * lg;
    const float phi = 2 * kPi * u2;
    const float c = 1 / sqrtf(1 + t2);
    const float s = sqrtf(fmaxf(0.f, 1 - c * c));
    float sn, cs;
    sincosf(phi, &sn, &cs);
    V3 h = v3(s * cs, s * sn, c);
    if (!(wo.z * h.z > 0)) h = -h;
    return h;
}
// BeckmannBSDF::lightReflected (BeckmannBSDF.cu:53-87), |cos wi| included
__device__ __forceinline__ V3 beckmann_eval(const Ggx &g, V3 kd, V3 eta, V3 k, V3 wo, V3 wi)
{
    if (!(wo.z * wi.z > 0)) return v3(0, 0, 0);
    if (fmaxf(g.ax, g.ay) < 1e-3f) return v3(0, 0, 0);
    const float co = abs_cos(wo), ci = abs_cos(wi);
    V3 h = wi + wo;
    if (ci == 0 || co == 0) return v3(0, 0, 0);
    if (h.x == 0 && h.y == 0 && h.z == 0) return v3(0, 0, 0);
    h = normalize(h);
    const float c = dot(wi, h) / (length(wi) * length(h));
    const V3 F = v3(fresnel_conductor(c, eta.x, k.x), fresnel_conductor(c, eta.y, k.y), fresnel_conductor(c, eta.z, k.z));
    const float D = beckmann_D(h, g.ax, g.ay);
    const float G = 1 / (1 + beckmann_lambda(wo, g.ax, g.ay) + beckmann_lambda(wi, g.ax, g.ay));
    return kd * D * G * F * (1.0f / (4 * ci * co)) * ci;
}
// BeckmannBSDF::pdf (BeckmannBSDF.cu:118-122): D(h) |cos h| / (4 |cos(wo, h)|) at the
// unnormalised h = wi + wo
__device__ __forceinline__ float beckmann_pdf(const Ggx &g, V3 wo, V3 wi)
{
    const V3 h = wi + wo;
    return beckmann_D(h, g.ax, g.ay) * abs_cos(h) / (4 * abs_cos2(wo, h));
}
// FresnelBlendMaterial::lightReflected (FresnelBlendMaterial.cu:111-135) with its kd = 1,
// ks = 0, alpha = 0.5: a diffuse lobe plus Schlick(R0 = 0) x Beckmann over
// 4 |cos(wi, h)| max(|cos wi|, |cos wo|); not weighted by |cos wi|
__device__ __forceinline__ V3 fresnel_blend_eval(V3 wo, V3 wi)
{
    auto pow5 = [](float x) { return (x * x) * (x * x) * x; };
    const float diffuse = (28.f / (23.f * kPi)) * (1 - pow5(1 - 0.5f * abs_cos(wi))) * (1 - pow5(1 - 0.5f * abs_cos(wo)));
    V3 h = wi + wo;
    if (h.x == 0 && h.y == 0 && h.z == 0) return v3(0, 0, 0);
    h = normalize(h);
    const float num = pow5(1 - dot(wi, h) / (length(wi) * length(h))) * beckmann_D(h, 0.5f, 0.5f);
    const float denom = 4 * abs_cos2(wi, h) * fmaxf(abs_cos(wi), abs_cos(wo));
    const float s = diffuse + num / denom;
    return v3(s, s, s);
}
// FresnelBlendMaterial::pdf (FresnelBlendMaterial.cu:137-141): D(h) |cos h| at h = wi + wo
__device__ __forceinline__ float fresnel_blend_pdf(V3 wo, V3 wi)
{
    const V3 h = wi + wo;
    return beckmann_D(h, 0.5f, 0.5f) * abs_cos(h);
}

// ------------------------------------------------------------- ONB / frames

// Orthonormal basis around n (Duff et al. 2017, "Building an Orthonormal Basis, Revisited").
__device__ __forceinline__ void onb(V3 n, V3 &t, V3 &b)
{
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    t = v3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = v3(bb, sign + n.y * n.y * a, -n.y);
}

// nextFloatUp / nextFloatDown (cuda_libraries/math.cu:147-194)
__device__ __forceinline__ float next_up(float x)
{
    if (isinf(x) && x > 0) return x;
    if (x == -0.0f) x = 0.0f;
    uint32_t u = __float_as_uint(x);
    u = (x >= 0) ? u + 1 : u - 1;
    return __uint_as_float(u);
}
__device__ __forceinline__ float next_down(float x)
{
    if (isinf(x) && x < 0) return x;
    if (x == 0.0f) x = -0.0f;
    uint32_t u = __float_as_uint(x);
    u = (x > 0) ? u - 1 : u + 1;
    return __uint_as_float(u);
}

// SurfaceInteraction::spawnRay (transformations/SurfaceInteraction.cu:162-185)
__device__ __forceinline__ V3 spawn_origin(V3 p, V3 n, V3 perr, V3 w)
{
    float d = dot(vabs(n), perr);
    V3 off = n * d;
    if (dot(w, n) < 0) off = -off;
    V3 po = p + off;
    po.x = off.x > 0 ? next_up(po.x) : (off.x < 0 ? next_down(po.x) : po.x);
    po.y = off.y > 0 ? next_up(po.y) : (off.y < 0 ? next_down(po.y) : po.y);
    po.z = off.z > 0 ? next_up(po.z) : (off.z < 0 ? next_down(po.z) : po.z);
    return po;
}

}  // namespace rtb
