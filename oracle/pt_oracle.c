/*
 * Test infrastructure only: CPU restatement of the path-tracing estimator that the CUDA
 * wavefront renderer implements (the reference's bounce loop, integration/pathTracing.cu:
 * 33-138, 173-205, 284-490, with Scene::sampleDirectLight, Scene.cu:280-335, 468-585),
 * consuming the same PCG32 stream per (pixel, sample) in the same order, so a sample
 * traced here follows the same path as on the GPU up to float rounding.
 *
 * Intersections use the restated reference traversal (rt_oracle.c). Materials follow
 * materials/{Lambertian,Trowbridge,Dielectric,SpecularReflection,SpecularRefraction,
 * PerfectReflection,Light,Plain}*.cu as cited below.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rt_oracle.h"
#include "rt_oracle_internal.h"

#define PI_F 3.14159265358979323846f
#define INV_PI_F 0.31830988618379067154f

enum { M_LAMB = 0, M_GGX = 1, M_DIEL = 2, M_LIGHT = 3, M_MIRROR = 4, M_PLAIN = 5, M_PHONG = 6, M_SSS = 7 };
enum { F_NEE_AREA = 1, F_COMPAT = 2 };

typedef struct {
    float x, y, z;
} v3;
static v3 V(float x, float y, float z)
{
    v3 r = {x, y, z};
    return r;
}
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static v3 mul(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 vmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 cross3(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float len3(v3 a) { return sqrtf(dot3(a, a)); }
static v3 norm3(v3 a) { return mul(a, 1.0f / len3(a)); }
static v3 vabs3(v3 a) { return V(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
static int black(v3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
static float lum(v3 a) { return 0.212671f * a.x + 0.715160f * a.y + 0.072169f * a.z; } /* Spectrum.cu:67-75 */

/* PCG32, seeded per (pixel, sample) exactly like the CUDA renderer. */
typedef struct {
    uint64_t state, inc;
} pcg;
static uint32_t pcg_next(pcg *r)
{
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ull + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
static pcg pcg_init(uint32_t pixel, uint32_t sample, uint32_t seed)
{
    pcg r;
    r.state = 0u;
    r.inc = ((((uint64_t)sample << 32) | seed) << 1u) | 1u;
    pcg_next(&r);
    r.state += (uint64_t)pixel;
    pcg_next(&r);
    return r;
}
static float pcg_f(pcg *r) { return (float)(pcg_next(r) >> 8) * (1.0f / 16777216.0f); }

/* Sampling::concentricSampleDisk / cosineSampleHemisphere (sampling/Sampler.cu:12-36, 73-90) */
static void concentric(float u1, float u2, float *dx, float *dy)
{
    float ox = 2.0f * u1 - 1.0f, oy = 2.0f * u2 - 1.0f;
    if (ox == 0.f && oy == 0.f) {
        *dx = *dy = 0.f;
        return;
    }
    float r, th;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        th = (PI_F / 4) * (oy / ox);
    } else {
        r = oy;
        th = (PI_F / 2) - (PI_F / 4) * (ox / oy);
    }
    *dx = r * cosf(th);
    *dy = r * sinf(th);
}
static v3 cos_hemi(float u1, float u2)
{
    float x, y;
    concentric(u1, u2, &x, &y);
    return V(x, y, sqrtf(fmaxf(0.f, 1.f - x * x - y * y)));
}

/* fresnelDielectric as written in the reference (cuda_libraries/geometricMath.cu:202-240) */
static float fresnel_ref(float cosO, float ni, float nt)
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
static float fresnel_phys(float cosI, float etaI, float etaT)
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

/* fresnelConductor (geometricMath.cu:242-261) with complex eta + i k */
typedef struct {
    float re, im;
} cx;
static cx C(float re, float im)
{
    cx c = {re, im};
    return c;
}
static cx cadd(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static cx csub(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
static cx cmul(cx a, cx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static float cnorm(cx a) { return a.re * a.re + a.im * a.im; }
static cx cdiv(cx a, cx b)
{
    float s = 1.0f / (b.re * b.re + b.im * b.im);
    return C(s * (a.re * b.re + a.im * b.im), s * (a.im * b.re - a.re * b.im));
}
static cx csqrt_(cx z)
{
    float m = sqrtf(cnorm(z));
    float re = sqrtf(fmaxf(0.f, 0.5f * (m + z.re)));
    float im = sqrtf(fmaxf(0.f, 0.5f * (m - z.re)));
    return C(re, z.im < 0 ? -im : im);
}
static float fresnel_cond(float cosI, float eta, float k)
{
    cosI = fminf(fmaxf(cosI, 0.f), 1.f);
    float sin2 = 1 - cosI * cosI;
    cx e = C(eta, k);
    cx sin2T = cdiv(C(sin2, 0.f), cmul(e, e));
    cx cosT = csqrt_(csub(C(1.f, 0.f), sin2T));
    cx ec = cmul(e, C(cosI, 0.f));
    cx rpar = cdiv(csub(ec, cosT), cadd(ec, cosT));
    cx ect = cmul(e, cosT);
    cx rper = cdiv(csub(C(cosI, 0.f), ect), cadd(C(cosI, 0.f), ect));
    return (cnorm(rpar) + cnorm(rper)) / 2;
}

/* Trowbridge-Reitz (materials/TrowbridgeBSDF.cu:12-253) */
static float c2t(v3 w) { return w.z * w.z; }
static float s2t(v3 w) { return fmaxf(0.f, 1 - c2t(w)); }
static float t2t(v3 w) { return s2t(w) / c2t(w); }
static float cphi(v3 w)
{
    float s = sqrtf(s2t(w));
    return s == 0 ? 1.f : fminf(fmaxf(w.x / s, -1.f), 1.f);
}
static float sphi(v3 w)
{
    float s = sqrtf(s2t(w));
    return s == 0 ? 0.f : fminf(fmaxf(w.y / s, -1.f), 1.f);
}
static float ggx_D(float ax, float ay, v3 h)
{
    float t2 = t2t(h);
    if (isinf(t2)) return 0.f;
    float c4 = c2t(h) * c2t(h);
    float cp = cphi(h) / ax, sp = sphi(h) / ay;
    float e = t2 * (cp * cp + sp * sp);
    return 1.0f / (PI_F * ax * ay * c4 * (1 + e) * (1 + e));
}
static float ggx_lambda(float ax, float ay, v3 w)
{
    float t2 = t2t(w);
    if (isinf(t2)) return 0.f;
    float cp = cphi(w) * ax, sp = sphi(w) * ay;
    return (sqrtf(1 + (cp * cp + sp * sp) * t2) - 1) / 2;
}
static float acos1(v3 w) { return fabsf(w.z / len3(w)); }
static float acos2(v3 a, v3 b) { return fabsf(dot3(a, b)) / (len3(a) * len3(b)); }
static float ggx_pdf_h(float ax, float ay, v3 wo, v3 h)
{
    return (1.0f / (1 + ggx_lambda(ax, ay, wo))) / acos1(wo) * ggx_D(ax, ay, h) * acos2(wo, h);
}
static v3 ggx_eval(float ax, float ay, v3 kd, v3 eta, v3 k, v3 wo, v3 wi)
{
    wo = norm3(wo);
    wi = norm3(wi);
    if (!(wo.z * wi.z > 0)) return V(0, 0, 0);
    if (fmaxf(ax, ay) < 1e-3f) return V(0, 0, 0);
    float co = acos1(wo), ci = acos1(wi);
    if (ci == 0 || co == 0) return V(0, 0, 0);
    v3 h = add(wi, wo);
    if (dot3(h, h) == 0) return V(0, 0, 0);
    h = norm3(h);
    float c = acos2(wo, h);
    v3 F = V(fresnel_cond(c, eta.x, k.x), fresnel_cond(c, eta.y, k.y), fresnel_cond(c, eta.z, k.z));
    float D = ggx_D(ax, ay, h);
    float G = 1.0f / (1 + ggx_lambda(ax, ay, wo) + ggx_lambda(ax, ay, wi));
    return mul(vmul(F, kd), (D * G / (4 * ci * co)) * ci);
}
static float ggx_pdf(float ax, float ay, v3 wo, v3 wi)
{
    if (!(wo.z * wi.z > 0)) return 0.f;
    if (fmaxf(ax, ay) < 1e-3f) return 0.f;
    v3 h = add(wo, wi);
    if (dot3(h, h) == 0) return 0.f;
    h = norm3(h);
    if (h.z < 0) h = neg(h);
    return ggx_pdf_h(ax, ay, wo, h) / (4 * acos2(wo, h));
}
static v3 ggx_sample_h(float ax, float ay, v3 wo, float u1, float u2)
{
    v3 wh = norm3(V(ax * wo.x, ay * wo.y, wo.z));
    if (wh.z < 0) wh = neg(wh);
    v3 T1 = (wh.z < 0.99999f) ? norm3(cross3(V(0, 0, 1), wh)) : V(1, 0, 0);
    v3 T2 = cross3(wh, T1);
    float sx = 2 * u1 - 1, sy = 2 * u2 - 1;
    float r = sqrtf(fabsf(sx)), th = 2 * PI_F * sy;
    float px = r * cosf(th), py = r * sinf(th);
    float hh = sqrtf(1 - px * px);
    float t = (1 + wh.z) / 2;
    py = (1 - t) * hh + t * py;
    float pz = sqrtf(fmaxf(0.f, 1 - (px * px + py * py)));
    v3 nh = add(add(mul(T1, px), mul(T2, py)), mul(wh, pz));
    return norm3(V(ax * nh.x, ay * nh.y, fmaxf(1e-6f, nh.z)));
}

static void onb(v3 n, v3 *t, v3 *b)
{
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    *t = V(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    *b = V(bb, sign + n.y * n.y * a, -n.y);
}

/* nextFloatUp/Down + spawnRay (cuda_libraries/math.cu:147-194, SurfaceInteraction.cu:162-185) */
static float nup(float x)
{
    if (isinf(x) && x > 0) return x;
    if (x == -0.0f) x = 0.0f;
    uint32_t u;
    memcpy(&u, &x, 4);
    u = (x >= 0) ? u + 1 : u - 1;
    memcpy(&x, &u, 4);
    return x;
}
static float ndown(float x)
{
    if (isinf(x) && x < 0) return x;
    if (x == 0.0f) x = -0.0f;
    uint32_t u;
    memcpy(&u, &x, 4);
    u = (x > 0) ? u - 1 : u + 1;
    memcpy(&x, &u, 4);
    return x;
}
static v3 spawn(v3 p, v3 n, v3 perr, v3 w)
{
    float d = dot3(vabs3(n), perr);
    v3 off = mul(n, d);
    if (dot3(w, n) < 0) off = neg(off);
    v3 po = add(p, off);
    po.x = off.x > 0 ? nup(po.x) : (off.x < 0 ? ndown(po.x) : po.x);
    po.y = off.y > 0 ? nup(po.y) : (off.y < 0 ? ndown(po.y) : po.y);
    po.z = off.z > 0 ? nup(po.z) : (off.z < 0 ? ndown(po.z) : po.z);
    return po;
}

static float eb(int n)
{
    double me = 5.9604644775390625e-08;
    return (float)((n * me) / (1 - n * me));
}

typedef struct {
    const rto_bvh *bvh;
    const uint32_t *tri_mat;
    const pto_sphere *sph;
    uint32_t nsph;
    const pto_material *mats;
    uint32_t nmat;
    const float *plights; /* 6 per light: position, I rgb */
    uint32_t npl;
    const pto_camera *cam;
    uint32_t spp, sample_offset, max_depth, rr_depth, seed, flags;
    /* emitters */
    uint32_t *etri;
    float *ecdf;
    uint32_t nemit;
    float etotal;
    double *sum;
    uint32_t *count;
    uint32_t pix_begin, pix_end;
} ctx_t;

static float maxc3(const float *c) { return fmaxf(c[0], fmaxf(c[1], c[2])); }
/* Material::isScattering / isSpecular; Phong and subsurface: kd, ks not black
 * (PhongMaterial.cu:45-58, SSMaterial.cu:55-58) */
static int is_scat(const pto_material *m)
{
    if (m->type == M_PHONG || m->type == M_SSS) return maxc3(m->color) > 0.f;
    return m->type == M_LAMB || m->type == M_GGX || m->type == M_PLAIN;
}
static int is_spec(const pto_material *m)
{
    if (m->type == M_PHONG) return maxc3(m->k) > 0.f;
    return m->type == M_GGX || m->type == M_DIEL;
}

/* closest hit: triangles (reference order) then spheres (Scene::intersects, Scene.cu:108-150) */
static int32_t closest(const ctx_t *c, v3 o, v3 d, float tmax, int shadow, float *t, float *b1, float *b2)
{
    float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    float tt = INFINITY;
    int32_t id = -1;
    *b1 = *b2 = 0.f;
    if (c->bvh) {
        rto_trace_one_full(c->bvh, oo, dd, tmax, shadow, &id, &tt, b1, b2);
        if (id < 0) tt = INFINITY;
    }
    for (uint32_t s = 0; s < c->nsph; s++) {
        if (shadow && (c->mats[c->sph[s].material].flags & 1u)) continue;
        float ts = tt;
        if (rto_sphere_intersects(c->sph[s].w2o, c->sph[s].radius, oo, dd, tmax, &ts)) {
            tt = ts;
            id = 0x40000000 | (int32_t)s;
            *b1 = *b2 = 0.f;
        }
    }
    *t = tt;
    return id;
}

static int occluded(const ctx_t *c, v3 o, v3 d, float tmax, int skip_transparent)
{
    float t, b1, b2;
    int32_t id = closest(c, o, d, tmax, skip_transparent, &t, &b1, &b2);
    return id >= 0 && t < tmax;
}

static v3 xpoint(const float *m, v3 p)
{
    float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
    float iw = 1.0f / w;
    return V(x * iw, y * iw, z * iw);
}
static v3 xvec(const float *m, v3 v)
{
    return V(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
             m[8] * v.x + m[9] * v.y + m[10] * v.z);
}

static v3 mat_color(const pto_material *m) { return V(m->color[0], m->color[1], m->color[2]); }

/* PhongMaterial::lightReflected (PhongMaterial.cu:70-88): Lambertian term plus
 * ks * max(0, cos(wo, mirror of wi))^ns when wi is above the surface */
static v3 phong_eval(const pto_material *m, v3 wo, v3 wi)
{
    v3 f = mul(mat_color(m), INV_PI_F * acos1(wi));
    if (wi.z / len3(wi) > 0.f) {
        v3 r = V(-wi.x, -wi.y, wi.z);
        float c = dot3(wo, r) / (len3(wo) * len3(r));
        f = add(f, mul(V(m->k[0], m->k[1], m->k[2]), powf(fmaxf(0.f, c), m->roughness[0])));
    }
    return f;
}

static v3 bsdf_eval(const pto_material *m, v3 wo, v3 wi, float *pdf)
{
    *pdf = 0.f;
    if (m->type == M_PHONG || m->type == M_SSS) { /* PhongMaterial::pdf: cosine(wi) / pi */
        *pdf = (wo.z * wi.z > 0) ? wi.z / len3(wi) * INV_PI_F : 0.f;
        return phong_eval(m, wo, wi);
    }
    if (m->type == M_LAMB) {
        *pdf = (wo.z * wi.z > 0) ? fabsf(wi.z) * INV_PI_F : 0.f;
        return mul(mat_color(m), INV_PI_F * acos1(wi));
    }
    if (m->type == M_GGX) {
        float ax = sqrtf(m->roughness[0]), ay = sqrtf(m->roughness[1]);
        *pdf = ggx_pdf(ax, ay, wo, wi);
        return ggx_eval(ax, ay, mat_color(m), V(m->eta[0], m->eta[1], m->eta[2]), V(m->k[0], m->k[1], m->k[2]), wo,
                        wi);
    }
    return V(0, 0, 0);
}

static v3 bsdf_sample(const pto_material *m, v3 wo, pcg *r, int compat, v3 *wi, float *pdf, int *delta)
{
    *delta = 0;
    *pdf = 0.f;
    v3 col = mat_color(m);
    switch (m->type) {
    case M_LAMB: {
        float u1 = pcg_f(r), u2 = pcg_f(r);
        *wi = cos_hemi(u1, u2);
        *pdf = wi->z * INV_PI_F;
        return col;
    }
    case M_GGX: {
        float u1 = pcg_f(r), u2 = pcg_f(r);
        float ax = sqrtf(m->roughness[0]), ay = sqrtf(m->roughness[1]);
        v3 eta = V(m->eta[0], m->eta[1], m->eta[2]), k = V(m->k[0], m->k[1], m->k[2]);
        v3 won = norm3(wo);
        if (fmaxf(ax, ay) < 1e-3f) {
            *wi = V(-won.x, -won.y, won.z);
            *delta = 1;
            float c = acos1(*wi);
            v3 F = V(fresnel_cond(c, eta.x, k.x), fresnel_cond(c, eta.y, k.y), fresnel_cond(c, eta.z, k.z));
            return mul(F, 1.0f / c);
        }
        v3 h = ggx_sample_h(ax, ay, won, u1, u2);
        *wi = sub(mul(h, 2 * dot3(won, h)), won);
        *pdf = ggx_pdf_h(ax, ay, won, h) / (4 * acos2(won, h));
        v3 f = ggx_eval(ax, ay, col, eta, k, won, *wi);
        if (!(*pdf > 0)) return V(0, 0, 0);
        return mul(f, 1.0f / *pdf);
    }
    case M_DIEL: {
        *delta = 1;
        float u = pcg_f(r);
        float c = wo.z / len3(wo);
        if (compat) {
            if (u < 0.7f) {
                float ni = 1.f, nt = m->ior;
                if (c < 0) {
                    float t = ni;
                    ni = nt;
                    nt = t;
                }
                float eta = ni / nt;
                v3 n = (wo.z < 0.f) ? V(0, 0, -1) : V(0, 0, 1);
                float co = dot3(n, wo) / len3(wo);
                float s2o = fmaxf(0.f, 1.f - co * co);
                float s2 = eta * eta * s2o;
                if (s2 >= 1) return V(0, 0, 0);
                float ct = sqrtf(1 - s2);
                *wi = add(mul(neg(wo), eta), mul(n, eta * co - ct));
                return mul(col, 1 - fresnel_ref(co, ni, nt));
            }
            *wi = V(-wo.x, -wo.y, wo.z);
            return mul(col, fresnel_ref(wi->z / len3(*wi), 1.f, m->ior));
        }
        float F = fresnel_phys(c, 1.f, m->ior);
        if (u < F) {
            *wi = V(-wo.x, -wo.y, wo.z);
            return col;
        }
        float ni = 1.f, nt = m->ior;
        v3 n = V(0, 0, 1);
        if (c < 0) {
            ni = m->ior;
            nt = 1.f;
            n = V(0, 0, -1);
        }
        float eta = ni / nt;
        float co = dot3(n, wo) / len3(wo);
        float s2 = eta * eta * fmaxf(0.f, 1.f - co * co);
        float ct = sqrtf(fmaxf(0.f, 1 - s2));
        *wi = add(mul(neg(wo), eta), mul(n, eta * co - ct));
        return col;
    }
    case M_PHONG:
    case M_SSS: { /* PhongMaterial::sampleDirection (PhongMaterial.cu:102-118) */
        float u1 = pcg_f(r), u2 = pcg_f(r);
        *wi = cos_hemi(u1, u2);
        *pdf = wi->z / len3(*wi) * INV_PI_F;
        if (!(*pdf > 0)) return V(0, 0, 0);
        return mul(phong_eval(m, wo, *wi), 1.0f / *pdf);
    }
    case M_MIRROR:
        *delta = 1;
        *wi = V(-wo.x, -wo.y, wo.z);
        return col;
    default:
        *wi = V(0, 0, 0);
        return V(0, 0, 0);
    }
}

static float emitter_pdf(const ctx_t *c, v3 Le, float dist2, float cosl)
{
    if (!(cosl > 0) || c->etotal <= 0) return 0.f;
    return lum(Le) / c->etotal * dist2 / cosl;
}

/* One camera sample (pixel, j): returns its radiance. */
static v3 trace_sample(const ctx_t *c, uint32_t pix, uint32_t j)
{
    const pto_camera *cam = c->cam;
    const uint32_t W = cam->width, H = cam->height;
    const int compat = (c->flags & F_COMPAT) != 0;
    const int nee_area = (c->flags & F_NEE_AREA) != 0 && c->nemit > 0;
    uint32_t px = pix % W, py = pix / W;
    pcg r = pcg_init(pix, j, c->seed);
    float fx = fminf(fmaxf((float)px + pcg_f(&r), 0.f), (float)W);
    float fy = fminf(fmaxf((float)py + pcg_f(&r), 0.f), (float)H);
    float l1 = pcg_f(&r), l2 = pcg_f(&r);
    v3 pc = xpoint(cam->raster_to_camera, V(fx, fy, 0.f));
    v3 oc = V(0, 0, 0), dc = norm3(pc);
    if (cam->lens_radius > 0) {
        float lx, ly;
        concentric(l1, l2, &lx, &ly);
        lx *= cam->lens_radius;
        ly *= cam->lens_radius;
        float ft = cam->focal_distance / pc.z;
        v3 pf = mul(pc, ft);
        oc = V(lx, ly, 0);
        dc = norm3(sub(pf, oc));
    }
    v3 o = xpoint(cam->camera_to_world, oc);
    v3 d = norm3(xvec(cam->camera_to_world, dc));
    v3 beta = V(1, 1, 1), L = V(0, 0, 0);
    float last_pdf = 0.f;
    int last_spec = 0, camera = 1;
    for (uint32_t depth = 0; depth < c->max_depth; depth++) {
        float t, b1, b2;
        int32_t prim = closest(c, o, d, INFINITY, 0, &t, &b1, &b2);
        if (prim < 0) break;
        v3 P, n, perr;
        uint32_t mid;
        int tri = !(prim & 0x40000000);
        float area_cos = 0.f;
        if (!tri) {
            const pto_sphere *s = &c->sph[prim & ~0x40000000];
            v3 ctr = V(s->o2w[3], s->o2w[7], s->o2w[11]);
            v3 p = add(o, mul(d, t));
            n = norm3(sub(p, ctr));
            P = add(ctr, mul(n, s->radius));
            perr = mul(add(vabs3(sub(P, ctr)), vabs3(ctr)), eb(5));
            mid = s->material;
        } else {
            float vv[9];
            rto_triangle_vertices(c->bvh, (uint32_t)prim, vv);
            v3 p0 = V(vv[0], vv[1], vv[2]), p1 = V(vv[3], vv[4], vv[5]), p2 = V(vv[6], vv[7], vv[8]);
            float b0 = 1.f - b1 - b2;
            P = add(add(mul(p0, b0), mul(p1, b1)), mul(p2, b2));
            v3 ng = norm3(cross3(sub(p0, p2), sub(p1, p2)));
            if (dot3(ng, d) > 0) ng = neg(ng);
            n = ng;
            perr = mul(add(add(vabs3(mul(p0, b0)), vabs3(mul(p1, b1))), vabs3(mul(p2, b2))), eb(7));
            mid = c->tri_mat[prim];
            area_cos = fabsf(dot3(ng, d));
        }
        if (mid >= c->nmat) mid = c->nmat - 1;
        const pto_material *m = &c->mats[mid];
        v3 tt, bb;
        onb(n, &tt, &bb);
        v3 wow = neg(d);
        v3 wo = V(dot3(wow, tt), dot3(wow, bb), dot3(wow, n));
        int scat = is_scat(m);
        v3 beta_in = beta;
        v3 Le = V(0, 0, 0);
        if (m->type == M_LIGHT)
            Le = mul(mat_color(m), m->intensity);
        else if (m->type == M_PLAIN && camera)
            Le = mat_color(m);
        if (!black(Le)) {
            float w = 1.f;
            if (nee_area && m->type == M_LIGHT && depth > 0 && !last_spec && tri) {
                float pl = emitter_pdf(c, Le, t * t, area_cos);
                w = (last_pdf * last_pdf) / (last_pdf * last_pdf + pl * pl);
            }
            L = add(L, mul(vmul(beta_in, Le), w));
        }
        v3 wil;
        float pdfb;
        int delta;
        v3 f = bsdf_sample(m, wo, &r, compat, &wil, &pdfb, &delta);
        v3 wiw = add(add(mul(tt, wil.x), mul(bb, wil.y)), mul(n, wil.z));
        beta = vmul(beta, f);
        int finished = black(f);
        if (!finished && scat && depth > c->rr_depth) {
            /* the reference's brightness (luminance) in compat mode; the largest component
             * otherwise, so no channel's throughput grows past 1 by surviving */
            float q = fmaxf(0.05f, 1.f - (compat ? lum(beta) : fmaxf(beta.x, fmaxf(beta.y, beta.z))));
            if (pcg_f(&r) < q)
                finished = 1;
            else
                beta = mul(beta, 1.f / (1.f - q));
        }
        if (!finished && depth + 1 >= c->max_depth) finished = 1;
        if (scat) {
            for (uint32_t li = 0; li < c->npl; li++) {
                const float *lp = c->plights + 6 * li;
                v3 tol = sub(V(lp[0], lp[1], lp[2]), P);
                float dist2 = dot3(tol, tol), dist = sqrtf(dist2);
                v3 wl = mul(tol, 1.0f / dist);
                (void)pcg_f(&r);
                (void)pcg_f(&r);
                if (!(dot3(wl, n) > 0)) continue;
                v3 wls = V(dot3(wl, tt), dot3(wl, bb), dot3(wl, n));
                float pb;
                v3 fl = bsdf_eval(m, wo, wls, &pb);
                v3 Li = mul(V(lp[3], lp[4], lp[5]), 1.0f / dist2);
                if (black(fl) || black(Li)) continue;
                float w = compat ? 1.0f / (1.0f + pb * pb) : 1.0f;
                v3 cc = mul(vmul(vmul(beta_in, fl), Li), w);
                if (!occluded(c, spawn(P, n, perr, wl), wl, dist, compat)) L = add(L, cc);
            }
            if (nee_area) {
                float u0 = pcg_f(&r), u1 = pcg_f(&r), u2 = pcg_f(&r);
                float x = u0 * c->etotal;
                uint32_t lo = 0, hi = c->nemit - 1;
                while (lo < hi) {
                    uint32_t mid2 = (lo + hi) >> 1;
                    if (c->ecdf[mid2] <= x)
                        lo = mid2 + 1;
                    else
                        hi = mid2;
                }
                uint32_t et = c->etri[lo];
                float ev[9];
                rto_triangle_vertices(c->bvh, et, ev);
                v3 e0 = V(ev[0], ev[1], ev[2]), e1 = V(ev[3], ev[4], ev[5]), e2 = V(ev[6], ev[7], ev[8]);
                float su = sqrtf(u1);
                float c0 = 1 - su, c1 = u2 * su;
                v3 xl = add(add(mul(e0, c0), mul(e1, c1)), mul(e2, 1 - c0 - c1));
                v3 nl = norm3(cross3(sub(e1, e0), sub(e2, e0)));
                v3 tol = sub(xl, P);
                float dist2 = dot3(tol, tol), dist = sqrtf(dist2);
                v3 wl = mul(tol, 1.0f / dist);
                float cosl = fabsf(dot3(nl, wl));
                uint32_t emid = c->tri_mat[et] < c->nmat ? c->tri_mat[et] : c->nmat - 1;
                const pto_material *em = &c->mats[emid];
                v3 Lel = mul(mat_color(em), em->intensity);
                float pl = emitter_pdf(c, Lel, dist2, cosl);
                if (pl > 0 && dot3(wl, n) > 0) {
                    v3 wls = V(dot3(wl, tt), dot3(wl, bb), dot3(wl, n));
                    float pb;
                    v3 fl = bsdf_eval(m, wo, wls, &pb);
                    if (!black(fl)) {
                        float w = (pl * pl) / (pl * pl + pb * pb);
                        v3 cc = mul(vmul(vmul(beta_in, fl), Lel), w / pl);
                        if (!occluded(c, spawn(P, n, perr, wl), wl, dist * (1.0f - 1e-4f), 0)) L = add(L, cc);
                    }
                }
            }
        }
        if (finished) break;
        o = spawn(P, n, perr, wiw);
        d = wiw;
        last_pdf = delta ? 0.f : pdfb;
        last_spec = delta;
        camera = camera && is_spec(m);
    }
    return L;
}

static void *worker(void *arg)
{
    ctx_t *c = (ctx_t *)arg;
    for (uint32_t pix = c->pix_begin; pix < c->pix_end; pix++) {
        for (uint32_t k = 0; k < c->spp; k++) {
            v3 L = trace_sample(c, pix, c->sample_offset + k);
            if (!(isfinite(L.x) && isfinite(L.y) && isfinite(L.z))) continue;
            c->sum[3 * (size_t)pix] += L.x;
            c->sum[3 * (size_t)pix + 1] += L.y;
            c->sum[3 * (size_t)pix + 2] += L.z;
            c->count[pix]++;
        }
    }
    return NULL;
}

int pto_render(const rto_bvh *bvh, const uint32_t *tri_mat, const pto_sphere *sph, uint32_t nsph,
               const pto_material *mats, uint32_t nmat, const float *plights, uint32_t npl, const pto_camera *cam,
               uint32_t spp, uint32_t sample_offset, uint32_t max_depth, uint32_t rr_depth, uint32_t seed,
               uint32_t flags, uint32_t pix_begin, uint32_t pix_end, double *sum, uint32_t *count, int nthreads)
{
    ctx_t base;
    memset(&base, 0, sizeof(base));
    base.bvh = bvh;
    base.tri_mat = tri_mat;
    base.sph = sph;
    base.nsph = nsph;
    base.mats = mats;
    base.nmat = nmat;
    base.plights = plights;
    base.npl = npl;
    base.cam = cam;
    base.spp = spp;
    base.sample_offset = sample_offset;
    base.max_depth = max_depth;
    base.rr_depth = rr_depth;
    base.seed = seed;
    base.flags = flags;
    base.sum = sum;
    base.count = count;
    /* emitters: area * luminance(Le), in triangle order (the renderer's CDF) */
    uint32_t ntri = bvh ? rto_bvh_ntri(bvh) : 0;
    base.etri = (uint32_t *)malloc(sizeof(uint32_t) * (ntri + 1));
    base.ecdf = (float *)malloc(sizeof(float) * (ntri + 1));
    double acc = 0;
    for (uint32_t t = 0; t < ntri; t++) {
        uint32_t mid = tri_mat[t] < nmat ? tri_mat[t] : nmat - 1;
        const pto_material *m = &mats[mid];
        if (m->type != M_LIGHT) continue;
        float p[9];
        rto_triangle_vertices(bvh, t, p);
        double ax = p[3] - p[0], ay = p[4] - p[1], az = p[5] - p[2];
        double bx = p[6] - p[0], by = p[7] - p[1], bz = p[8] - p[2];
        double cx_ = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
        double area = 0.5 * sqrt(cx_ * cx_ + cy * cy + cz * cz);
        double l = 0.212671 * m->color[0] * m->intensity + 0.715160 * m->color[1] * m->intensity +
                   0.072169 * m->color[2] * m->intensity;
        if (!(area * l > 0)) continue;
        acc += area * l;
        base.etri[base.nemit] = t;
        base.ecdf[base.nemit] = (float)acc;
        base.nemit++;
    }
    base.etotal = (float)acc;
    if (nthreads < 1) nthreads = 1;
    uint32_t npix = pix_end - pix_begin;
    if ((uint32_t)nthreads > npix) nthreads = (int)(npix ? npix : 1);
    ctx_t *cs = (ctx_t *)malloc(sizeof(ctx_t) * nthreads);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    for (int i = 0; i < nthreads; i++) {
        cs[i] = base;
        cs[i].pix_begin = pix_begin + (uint32_t)((uint64_t)npix * i / nthreads);
        cs[i].pix_end = pix_begin + (uint32_t)((uint64_t)npix * (i + 1) / nthreads);
        pthread_create(&th[i], NULL, worker, &cs[i]);
    }
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    free(cs);
    free(th);
    free(base.etri);
    free(base.ecdf);
    return 0;
}


/* ------------------------------------------------------------------ photons */

/* Photon tracing with the renderer's per-photon PCG streams (Scene::generatePhotons,
 * Scene.cu:989-1018; PointLight::sampleLight, PointLight.cu:68-95; computePhotons /
 * samplePhotonIntersections, photonDispersion.cu:26-172). Output photons in (path, depth)
 * order, 16 floats each: pos[3], shape, dir[3], path, power[3], depth, normal[3], 0. */
uint64_t pto_trace_photons(const rto_bvh *bvh, const uint32_t *tri_mat, const int32_t *tri_shape,
                           const pto_sphere *sph, const int32_t *sph_shape, uint32_t nsph, const pto_material *mats,
                           uint32_t nmat, const float *plights, const float *plight_rgbi, uint32_t npl, uint64_t n,
                           uint32_t max_depth, uint32_t rr_depth, uint32_t seed, uint32_t flags, float *out,
                           uint64_t cap)
{
    ctx_t c;
    memset(&c, 0, sizeof(c));
    c.bvh = bvh;
    c.tri_mat = tri_mat;
    c.sph = sph;
    c.nsph = nsph;
    c.mats = mats;
    c.nmat = nmat;
    const int compat = (flags & F_COMPAT) != 0;
    float *power = (float *)malloc(sizeof(float) * npl);
    float total = 0.f;
    for (uint32_t l = 0; l < npl; l++) {
        const float *q = plight_rgbi + 4 * l;
        power[l] = (q[0] * q[3] * 4.0f * PI_F) + (q[1] * q[3] * 4.0f * PI_F) + (q[2] * q[3] * 4.0f * PI_F);
        total += power[l];
    }
    uint32_t *sel = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint64_t *perl = (uint64_t *)calloc(npl, sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++) {
        pcg r = pcg_init((uint32_t)i, 0xFFFFFFFFu, seed ^ 0x9E3779B9u);
        float u = pcg_f(&r);
        uint32_t l = npl - 1;
        for (uint32_t k = 0; k < npl; k++) {
            u -= power[k] / total;
            if (u <= 0) {
                l = k;
                break;
            }
        }
        sel[i] = l;
        perl[l]++;
    }
    uint64_t stored = 0;
    for (uint64_t i = 0; i < n; i++) {
        pcg r = pcg_init((uint32_t)i, 0xFFFFFFFFu, seed ^ 0x9E3779B9u);
        (void)pcg_f(&r);
        uint32_t l = sel[i];
        float u1 = pcg_f(&r), u2 = pcg_f(&r);
        float phi = 2 * PI_F * u1, th = acosf(2 * u2 - 1);
        v3 d = V(sinf(th) * cosf(phi), sinf(th) * sinf(phi), cosf(th));
        const float *lp = plights + 6 * l;
        float scale = (4 * PI_F) / (float)perl[l] / (power[l] / total);
        v3 carry = V(lp[3] * scale, lp[4] * scale, lp[5] * scale);
        v3 o = V(lp[0], lp[1], lp[2]);
        v3 beta = V(1, 1, 1);
        for (uint32_t depth = 0; depth < max_depth; depth++) {
            float t, b1, b2;
            int32_t prim = closest(&c, o, d, INFINITY, 0, &t, &b1, &b2);
            if (prim < 0) break;
            v3 P, nn, perr;
            uint32_t mid;
            int32_t shape;
            if (prim & 0x40000000) {
                uint32_t si = (uint32_t)(prim & ~0x40000000);
                const pto_sphere *sp = &sph[si];
                v3 ctr = V(sp->o2w[3], sp->o2w[7], sp->o2w[11]);
                v3 p = add(o, mul(d, t));
                nn = norm3(sub(p, ctr));
                P = add(ctr, mul(nn, sp->radius));
                perr = mul(add(vabs3(sub(P, ctr)), vabs3(ctr)), eb(5));
                mid = sp->material;
                shape = sph_shape[si];
            } else {
                float vv[9];
                rto_triangle_vertices(bvh, (uint32_t)prim, vv);
                v3 p0 = V(vv[0], vv[1], vv[2]), p1 = V(vv[3], vv[4], vv[5]), p2 = V(vv[6], vv[7], vv[8]);
                float b0 = 1.f - b1 - b2;
                P = add(add(mul(p0, b0), mul(p1, b1)), mul(p2, b2));
                v3 ng = norm3(cross3(sub(p0, p2), sub(p1, p2)));
                if (dot3(ng, d) > 0) ng = neg(ng);
                nn = ng;
                perr = mul(add(add(vabs3(mul(p0, b0)), vabs3(mul(p1, b1))), vabs3(mul(p2, b2))), eb(7));
                mid = tri_mat[prim];
                shape = tri_shape[prim];
            }
            if (mid >= nmat) mid = nmat - 1;
            const pto_material *m = &mats[mid];
            if (is_scat(m)) {
                if (stored < cap) {
                    float *ph = out + 16 * stored;
                    v3 pw = vmul(carry, beta);
                    uint32_t u32;
                    ph[0] = P.x, ph[1] = P.y, ph[2] = P.z;
                    memcpy(&ph[3], &shape, 4);
                    ph[4] = d.x, ph[5] = d.y, ph[6] = d.z;
                    u32 = (uint32_t)i;
                    memcpy(&ph[7], &u32, 4);
                    ph[8] = pw.x, ph[9] = pw.y, ph[10] = pw.z;
                    memcpy(&ph[11], &depth, 4);
                    ph[12] = nn.x, ph[13] = nn.y, ph[14] = nn.z, ph[15] = 0.f;
                }
                stored++;
            }
            v3 tt, bb;
            onb(nn, &tt, &bb);
            v3 wow = neg(d);
            v3 wo = V(dot3(wow, tt), dot3(wow, bb), dot3(wow, nn));
            v3 Le = (m->type == M_LIGHT) ? mul(mat_color(m), m->intensity) : V(0, 0, 0);
            v3 wil;
            float pdfb;
            int delta;
            v3 f = bsdf_sample(m, wo, &r, compat, &wil, &pdfb, &delta);
            carry = add(carry, vmul(beta, Le));
            beta = vmul(beta, f);
            int finished = black(f);
            if (!finished && is_scat(m) && depth > rr_depth) {
                float q = fmaxf(0.05f, 1.f - lum(beta));
                if (pcg_f(&r) < q)
                    finished = 1;
                else
                    beta = mul(beta, 1.f / (1.f - q));
            }
            if (finished || depth + 1 >= max_depth) break;
            v3 wiw = add(add(mul(tt, wil.x), mul(bb, wil.y)), mul(nn, wil.z));
            o = spawn(P, nn, perr, wiw);
            d = wiw;
        }
    }
    free(power);
    free(sel);
    free(perl);
    return stored;
}


/* The Phong BSDF of the estimator (eval and pdf) for n shading-space direction pairs. */
void pto_phong_eval(const pto_material *m, const float *wo, const float *wi, uint32_t n, float *out_f, float *out_pdf)
{
    for (uint32_t i = 0; i < n; i++) {
        float pdf;
        v3 f = bsdf_eval(m, V(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), V(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), &pdf);
        out_f[3 * i] = f.x;
        out_f[3 * i + 1] = f.y;
        out_f[3 * i + 2] = f.z;
        out_pdf[i] = pdf;
    }
}
