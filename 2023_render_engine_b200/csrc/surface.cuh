// Surface reconstruction, materials and BSDF sampling shared by the path tracer
// (render.cu) and the photon tracer (photon.cu).
#pragma once

#include <cooperative_groups.h>

#include "shading.cuh"
#include "traverse.cuh"

namespace rtb {

namespace cg = cooperative_groups;

// Device view of everything shading needs.
struct RenderView {
    SceneView sv;
    const rt_material *mats;
    const uint32_t *tri_mat;
    const int32_t *tri_shape;  // shape id per triangle (the reference's meshId)
    const int32_t *tri_nidx;  // 3 per triangle, -1 when the mesh has no normals
    const float *normals;
    const uint32_t *emit_tri;
    const float *emit_cdf;
    uint32_t nemit;
    float emit_total;  // sum over emitters of area * luminance(Le)
    const float4 *plights;  // 2 per light: position, radiant intensity rgb
    uint32_t nplights;
    uint32_t nmats;
    // the views of the render (one for rt_render): camera and options, the first global
    // sample index of each view (nviews + 1 entries) and its first pixel in the films
    const rt_view *views;
    const uint64_t *view_sample0;
    const uint32_t *view_pixel0;
    uint32_t nviews;
    uint32_t flags;
    uint64_t total;  // samples over all views
    // textures: texels (rgb), per texture (first texel, width, height, 0); texture
    // coordinates, 6 per triangle (null: every triangle uses the default ones)
    const float4 *texels;
    const uint4 *tex_info;
    const float *tri_uv;
    uint32_t ntex;
};

// view of global sample g / of global film pixel p (binary search over the prefix sums)
__device__ __forceinline__ uint32_t view_of_sample(const RenderView &rv, uint64_t g)
{
    uint32_t lo = 0, hi = rv.nviews - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (rv.view_sample0[mid] <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ uint32_t view_of_pixel(const RenderView &rv, uint32_t p)
{
    uint32_t lo = 0, hi = rv.nviews - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (rv.view_pixel0[mid] <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Warp-aggregated queue append: one atomic per group of active lanes.
__device__ __forceinline__ uint32_t append(uint32_t *counter)
{
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

__device__ __forceinline__ V3 xform_point(const float *m, V3 p)
{
    float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
    float iw = 1.0f / w;
    return v3(x * iw, y * iw, z * iw);
}
__device__ __forceinline__ V3 xform_vec(const float *m, V3 v)
{
    return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
              m[8] * v.x + m[9] * v.y + m[10] * v.z);
}

struct Surface {
    V3 p, n, perr;  // position, shading normal (faces the ray for triangles), error bound
    uint32_t mat;
    int32_t shape;  // SurfaceInteraction::shapeId: mesh id for triangles, shape index for spheres
    bool emissive_tri;
    float area_cos;  // for MIS: |cos| at the emitter
};

// Triangle / sphere hit -> surface (Triangle::intersect, Triangle.cu:319-428;
// Sphere::intersect, Sphere.cu:277-355).
__device__ __forceinline__ Surface surface_at(const RenderView &rv, const rt_hit &h, V3 o, V3 d, bool compat)
{
    Surface s;
    if (h.prim & RT_PRIM_SHAPE) {
        const SphereRecord &sr = rv.sv.spheres[h.prim & ~RT_PRIM_SHAPE];
        if (sr.flags & kShapePlane) {
            // Plane::intersect (Plane.cu:62-122): the object-space hit (x, y, 0) the trace reports
            // in (b1, b2) carried to world space; the normal (0, 0, 1) turned against the ray; the
            // reference's fixed object-space error bound 1e-4 carried by the transform
            const float *m = sr.o2w;
            const V3 lp = v3(h.b1, h.b2, 0.f);
            s.p = xform_point(m, lp);
            V3 n = normalize(v3(sr.w2o[8], sr.w2o[9], sr.w2o[10]));
            if (dot(n, d) > 0) n = -n;
            s.n = n;
            const float eb3 = error_bound(3);
            const V3 rows = v3(fabsf(m[0]) + fabsf(m[1]) + fabsf(m[2]), fabsf(m[4]) + fabsf(m[5]) + fabsf(m[6]),
                               fabsf(m[8]) + fabsf(m[9]) + fabsf(m[10]));
            const V3 mag = v3(fabsf(m[0] * lp.x) + fabsf(m[1] * lp.y) + fabsf(m[3]),
                              fabsf(m[4] * lp.x) + fabsf(m[5] * lp.y) + fabsf(m[7]),
                              fabsf(m[8] * lp.x) + fabsf(m[9] * lp.y) + fabsf(m[11]));
            s.perr = rows * (1e-4f * (1.f + eb3)) + mag * eb3;
            s.mat = sr.material;
            s.shape = sr.shape_id;
            s.emissive_tri = false;
            s.area_cos = 0.f;
            return s;
        }
        V3 c = v3(sr.o2w[3], sr.o2w[7], sr.o2w[11]);
        V3 p = o + d * h.t;
        V3 n = normalize(p - c);
        s.p = c + n * sr.radius;
        s.n = n;  // outward: -cross(dpdu, dpdv) of the reference parametrisation (Sphere.cu:159-160)
        const float eb5 = error_bound(5);
        s.perr = (vabs(s.p - c) + vabs(c)) * eb5;
        s.mat = sr.material;
        s.shape = sr.shape_id;
        s.emissive_tri = false;
        s.area_cos = 0.f;
        return s;
    }
    const TriRecord tr = rv.sv.tris[rv.sv.leafpos[h.prim]];
    V3 p0 = v3(tr.v0.x, tr.v0.y, tr.v0.z), p1 = v3(tr.v1.x, tr.v1.y, tr.v1.z), p2 = v3(tr.v2.x, tr.v2.y, tr.v2.z);
    float b1 = h.b1, b2 = h.b2, b0 = 1.f - b1 - b2;
    s.p = p0 * b0 + p1 * b1 + p2 * b2;
    V3 ng = normalize(cross(p0 - p2, p1 - p2));
    if (dot(ng, d) > 0) ng = -ng;  // Triangle.cu:370-373
    s.n = ng;
    const float eb7 = error_bound(7);
    s.perr = (vabs(p0 * b0) + vabs(p1 * b1) + vabs(p2 * b2)) * eb7;
    if (rv.tri_nidx && rv.tri_nidx[3 * h.prim] >= 0) {
        const int32_t *ni = rv.tri_nidx + 3 * h.prim;
        V3 n0 = v3(rv.normals[3 * ni[0]], rv.normals[3 * ni[0] + 1], rv.normals[3 * ni[0] + 2]);
        V3 n1 = v3(rv.normals[3 * ni[1]], rv.normals[3 * ni[1] + 1], rv.normals[3 * ni[1] + 2]);
        V3 n2 = v3(rv.normals[3 * ni[2]], rv.normals[3 * ni[2] + 1], rv.normals[3 * ni[2] + 2]);
        V3 ns = normalize(n0 * b0 + n1 * b1 + n2 * b2);
        s.n = ns;
        if (compat) s.p = s.p + ns * 0.15f;  // Triangle.cu:418
    }
    s.mat = rv.tri_mat[h.prim];
    s.shape = rv.tri_shape ? rv.tri_shape[h.prim] : 0;
    s.emissive_tri = true;
    s.area_cos = fabsf(dot(ng, d));
    return s;
}

// ------------------------------------------------------------------ textures

// Texel index along one axis as Texture::getColor computes it (Texture.cu:179-192):
// `unsigned int x = point.x * getWidth()` converts the float product the way the reference's
// x86-64 build does (truncation to a 64-bit integer, low 32 bits kept; NaN and out-of-range
// values give 0), then clamp(x, 0, size - 1) picks the float overload of clamp, which for
// these non-negative values is min(x, size - 1).
__host__ __device__ __forceinline__ uint32_t tex_index(float c, uint32_t size)
{
    const float x = c * (float)size;
    const long long i = (fabsf(x) < 9.22337204e18f) ? (long long)x : (long long)(1ull << 63);
    const uint32_t u = (uint32_t)(unsigned long long)i;
    return u < size - 1 ? u : size - 1;
}

// Texture::getColor of texture `id` at surface point (u, v): pixelMatrix[y][x]
__device__ __forceinline__ V3 tex_color(const RenderView &rv, uint32_t id, float u, float v)
{
    const uint4 t = rv.tex_info[id];
    const float4 c = rv.texels[t.x + (uint64_t)tex_index(v, t.z) * t.y + tex_index(u, t.y)];
    return v3(c.x, c.y, c.z);
}

// Surface point of a hit: the barycentric blend of the triangle's texture coordinates
// (Triangle.cu:355-358; without coordinates (0,0), (1,0), (1,1), Triangle.cu:134-151), or a
// sphere's (theta, phi) in degrees from its object-space hit point (Sphere::localToSurface,
// to_spherical, geometricMath.cu:49-57; degrees() rounds radians * 180.0 / PI in double).
__device__ __forceinline__ float2 surface_uv(const RenderView &rv, const rt_hit &h, const Surface &s)
{
    if (h.prim & RT_PRIM_SHAPE) {
        if (rv.sv.spheres[h.prim & ~RT_PRIM_SHAPE].flags & kShapePlane) return make_float2(h.b1, h.b2);  // Plane.cu:82
        const float *m = rv.sv.spheres[h.prim & ~RT_PRIM_SHAPE].w2o;
        const float x = m[0] * s.p.x + m[1] * s.p.y + m[2] * s.p.z + m[3];
        const float y = m[4] * s.p.x + m[5] * s.p.y + m[6] * s.p.z + m[7];
        const float z = m[8] * s.p.x + m[9] * s.p.y + m[10] * s.p.z + m[11];
        const float th = atan2f(sqrtf(x * x + y * y), z), ph = atan2f(y, x);
        const double deg = 180.0 / (double)3.14159265358979f;
        return make_float2((float)((double)th * deg), (float)((double)ph * deg));
    }
    const float b1 = h.b1, b2 = h.b2, b0 = 1.f - b1 - b2;
    if (!rv.tri_uv) return make_float2(b1 + b2, b2);  // (0,0) b0 + (1,0) b1 + (1,1) b2
    const float *t = rv.tri_uv + 6ull * (uint32_t)h.prim;
    return make_float2(b0 * t[0] + b1 * t[2] + b2 * t[4], b0 * t[1] + b1 * t[3] + b2 * t[5]);
}

struct Bsdf {
    uint32_t type;
    V3 color;
    Ggx g;
    V3 eta, k;
    float ior;
};

__device__ __forceinline__ Bsdf load_bsdf(const rt_material &m)
{
    Bsdf b;
    b.type = m.type;
    b.color = v3(m.color[0], m.color[1], m.color[2]);
    b.g.ax = sqrtf(m.roughness[0]);
    b.g.ay = sqrtf(m.roughness[1]);
    b.eta = v3(m.eta[0], m.eta[1], m.eta[2]);
    b.k = v3(m.k[0], m.k[1], m.k[2]);
    b.ior = m.ior;
    if (b.type == RT_MAT_PHONG || b.type == RT_MAT_SUBSURFACE) b.g.ax = m.roughness[0];  // ns, as given
    return b;
}

// The texel's effect on a material (the reference's materials read their Texture in these
// places only): Lambertian (LambertianBSDF.cu:22-28, 66-70), Phong and the surface of
// SSMaterial (through their LambertianBRDF, PhongMaterial.cu:95) and Plain's emission
// (PlainMaterial.cu:66-67) multiply kd by it; Trowbridge, TrowbridgeBasic and Beckmann replace
// kd with it (TrowbridgeBSDF.cu:167-169, TrowbridgeBasicBSDF.cu:167-169, BeckmannBSDF.cu:61-63).
// FresnelBlend's LambertianBRDF is never evaluated, so its texture has no effect.
__device__ __forceinline__ void texture_bsdf(Bsdf &b, V3 texel)
{
    switch (b.type) {
    case RT_MAT_LAMBERTIAN:
    case RT_MAT_PHONG:
    case RT_MAT_SUBSURFACE:
    case RT_MAT_PLAIN: b.color = b.color * texel; break;
    case RT_MAT_TROWBRIDGE:
    case RT_MAT_TROWBRIDGE_BASIC:
    case RT_MAT_BECKMANN: b.color = texel; break;
    default: break;
    }
}

// Phong and subsurface surfaces keep ks in Bsdf::k and the exponent ns in g.ax.
__device__ __forceinline__ bool is_phong(uint32_t type) { return type == RT_MAT_PHONG || type == RT_MAT_SUBSURFACE; }

// Material::isScattering: PhongMaterial / SSMaterial scatter when kd is not black
// (PhongMaterial.cu:45-48, SSMaterial.cu:55-58).
// FresnelBlendMaterial scatters (its kd is always 1, FresnelBlendMaterial.cu:33-36).
__device__ __forceinline__ bool is_scattering(const Bsdf &b)
{
    if (is_phong(b.type)) return fmaxf(b.color.x, fmaxf(b.color.y, b.color.z)) > 0.f;
    return b.type == RT_MAT_LAMBERTIAN || b.type == RT_MAT_TROWBRIDGE || b.type == RT_MAT_PLAIN ||
           b.type == RT_MAT_BECKMANN || b.type == RT_MAT_TROWBRIDGE_BASIC || b.type == RT_MAT_FRESNEL_BLEND ||
           b.type == RT_MAT_PLASTIC;
}
__device__ __forceinline__ bool is_specular(const Bsdf &b)
{
    // Material::isSpecular overrides; PhongMaterial: ks not black (PhongMaterial.cu:55-58);
    // Beckmann, TrowbridgeBasic and PlasticUnreal: true; FresnelBlend: its ks (0) not black
    if (b.type == RT_MAT_PHONG) return fmaxf(b.k.x, fmaxf(b.k.y, b.k.z)) > 0.f;
    return b.type == RT_MAT_TROWBRIDGE || b.type == RT_MAT_DIELECTRIC || b.type == RT_MAT_BECKMANN ||
           b.type == RT_MAT_TROWBRIDGE_BASIC || b.type == RT_MAT_PLASTIC;
}

// PhongMaterial::lightReflected (PhongMaterial.cu:70-88): the Lambertian term plus
// ks * max(0, cos(wo, mirror of wi))^ns when wi is above the surface (not weighted by cos).
__device__ __forceinline__ V3 phong_eval(const Bsdf &b, V3 wo, V3 wi)
{
    V3 f = b.color * (kInvPi * abs_cos(wi));
    if (wi.z / length(wi) > 0.f) {
        const V3 r = v3(-wi.x, -wi.y, wi.z);
        const float c = dot(wo, r) / (length(wo) * length(r));
        f = f + b.k * powf(fmaxf(0.f, c), b.g.ax);
    }
    return f;
}

// f * |cos wi| and pdf, shading space.
__device__ __forceinline__ V3 bsdf_eval(const Bsdf &b, V3 wo, V3 wi, float &pdf)
{
    pdf = 0.f;
    switch (b.type) {
    case RT_MAT_LAMBERTIAN:  // LambertianBSDF.cu:32-47: cosine(wi) / pi on wo's side (signed)
        pdf = (wo.z * wi.z > 0) ? wi.z / length(wi) * kInvPi : 0.f;
        return b.color * (kInvPi * abs_cos(wi));
    case RT_MAT_PHONG:
    case RT_MAT_SUBSURFACE:  // PhongMaterial::pdf: cosine(wi) / pi on wo's side (PhongMaterial.cu:94-100)
        pdf = (wo.z * wi.z > 0) ? wi.z / length(wi) * kInvPi : 0.f;
        return phong_eval(b, wo, wi);
    case RT_MAT_TROWBRIDGE:
        pdf = ggx_pdf(b.g, wo, wi);
        return ggx_eval(b.g, b.color, b.eta, b.k, wo, wi);
    case RT_MAT_TROWBRIDGE_BASIC:  // TrowbridgeBasicBSDF.cu:155-210
        pdf = ggx_pdf(b.g, wo, wi);
        return ggx_eval(b.g, b.color, b.eta, b.k, wo, wi, true);
    case RT_MAT_BECKMANN:  // BeckmannBSDF.cu:53-122
        pdf = beckmann_pdf(b.g, wo, wi);
        return beckmann_eval(b.g, b.color, b.eta, b.k, wo, wi);
    case RT_MAT_FRESNEL_BLEND:  // FresnelBlendMaterial.cu:111-141
        pdf = fresnel_blend_pdf(wo, wi);
        return fresnel_blend_eval(wo, wi);
    case RT_MAT_PLASTIC:  // PlasticUnrealMaterial.cu:49-59: the Lambertian lobe, pdf 0
        return b.color * (kInvPi * abs_cos(wi));
    default:
        return v3(0, 0, 0);
    }
}

// Samples wi; returns f*|cos|/pdf (the reference's sampleDirection value).
__device__ __forceinline__ V3 bsdf_sample(const Bsdf &b, V3 wo, Pcg &r, bool compat, V3 &wi, float &pdf, bool &delta)
{
    delta = false;
    pdf = 0.f;
    switch (b.type) {
    case RT_MAT_LAMBERTIAN: {  // LambertianBSDF.cu:56-75
        float u1 = pcg_float(r), u2 = pcg_float(r);
        wi = cosine_hemisphere(u1, u2);
        pdf = wi.z * kInvPi;
        return b.color;
    }
    case RT_MAT_TROWBRIDGE: {  // TrowbridgeBSDF.cu:207-246
        float u1 = pcg_float(r), u2 = pcg_float(r);
        V3 won = normalize(wo);
        if (fmaxf(b.g.ax, b.g.ay) < 1e-3f) {
            wi = v3(-won.x, -won.y, won.z);
            delta = true;
            float c = abs_cos(wi);
            V3 F = v3(fresnel_conductor(c, b.eta.x, b.k.x), fresnel_conductor(c, b.eta.y, b.k.y),
                      fresnel_conductor(c, b.eta.z, b.k.z));
            return F * (1.0f / c);
        }
        V3 h = ggx_sample_h(b.g, won, u1, u2);
        wi = h * (2 * dot(won, h)) - won;  // reflect (geometricMath.cu:197-200)
        pdf = ggx_pdf_h(b.g, won, h) / (4 * abs_cos2(won, h));
        V3 f = ggx_eval(b.g, b.color, b.eta, b.k, won, wi);
        if (!(pdf > 0)) return v3(0, 0, 0);
        return f * (1.0f / pdf);
    }
    case RT_MAT_DIELECTRIC: {
        delta = true;
        float u = pcg_float(r);
        float c = wo.z / length(wo);
        if (compat) {
            // DielectricMaterial.cu:59-77: refraction with probability 0.7, no division
            if (u < 0.7f) {  // SpecularRefractionBSDF.cu:31-63
                float ni = 1.f, nt = b.ior;
                if (c < 0) {
                    float t = ni;
                    ni = nt;
                    nt = t;
                }
                float eta = ni / nt;
                V3 n = (wo.z < 0.f) ? v3(0, 0, -1) : v3(0, 0, 1);
                float co = dot(n, wo) / length(wo);
                float s2o = fmaxf(0.f, 1.f - co * co);
                float s2t = eta * eta * s2o;
                if (s2t >= 1) return v3(0, 0, 0);
                float ct = sqrtf(1 - s2t);
                wi = (-wo) * eta + n * (eta * co - ct);
                return b.color * (1 - fresnel_dielectric_ref(co, ni, nt));
            }
            wi = v3(-wo.x, -wo.y, wo.z);  // SpecularReflectionBSDF.cu:30-41
            return b.color * fresnel_dielectric_ref(wi.z / length(wi), 1.f, b.ior);
        }
        float F = fresnel_dielectric(c, 1.f, b.ior);
        if (u < F) {
            wi = v3(-wo.x, -wo.y, wo.z);
            return b.color;
        }
        float ni = 1.f, nt = b.ior;
        V3 n = v3(0, 0, 1);
        if (c < 0) {
            ni = b.ior;
            nt = 1.f;
            n = v3(0, 0, -1);
        }
        float eta = ni / nt;
        float co = dot(n, wo) / length(wo);
        float s2t = eta * eta * fmaxf(0.f, 1.f - co * co);
        float ct = sqrtf(fmaxf(0.f, 1 - s2t));
        wi = (-wo) * eta + n * (eta * co - ct);
        return b.color;
    }
    case RT_MAT_PHONG:
    case RT_MAT_SUBSURFACE: {  // PhongMaterial::sampleDirection (PhongMaterial.cu:102-118)
        float u1 = pcg_float(r), u2 = pcg_float(r);
        wi = cosine_hemisphere(u1, u2);
        pdf = wi.z / length(wi) * kInvPi;
        if (!(pdf > 0)) return v3(0, 0, 0);
        return phong_eval(b, wo, wi) * (1.0f / pdf);
    }
    case RT_MAT_MIRROR:  // PerfectReflectionBSDF
        delta = true;
        wi = v3(-wo.x, -wo.y, wo.z);
        return b.color;
    case RT_MAT_TROWBRIDGE_BASIC: {  // TrowbridgeBasicBSDF.cu:213-246: Trowbridge with F = 1
        V3 won = normalize(wo);
        if (fmaxf(b.g.ax, b.g.ay) < 1e-3f) {
            wi = v3(-won.x, -won.y, won.z);
            delta = true;
            return v3(1, 1, 1);
        }
        float u1 = pcg_float(r), u2 = pcg_float(r);
        V3 h = ggx_sample_h(b.g, won, u1, u2);
        wi = h * (2 * dot(won, h)) - won;
        pdf = ggx_pdf_h(b.g, won, h) / (4 * abs_cos2(won, h));
        V3 f = ggx_eval(b.g, b.color, b.eta, b.k, won, wi, true);
        if (!(pdf > 0)) return v3(0, 0, 0);
        return f * (1.0f / pdf);
    }
    case RT_MAT_BECKMANN: {  // BeckmannBSDF.cu:125-148
        if (fmaxf(b.g.ax, b.g.ay) < 1e-3f) {
            wi = v3(-wo.x, -wo.y, wo.z);
            delta = true;
            const float c = abs_cos(wi);
            return v3(fresnel_conductor(c, b.eta.x, b.k.x), fresnel_conductor(c, b.eta.y, b.k.y),
                      fresnel_conductor(c, b.eta.z, b.k.z));
        }
        pcg_float(r);  // the reference draws a 2D sample it does not use
        pcg_float(r);
        const float u1 = pcg_float(r), u2 = pcg_float(r);
        const V3 h = beckmann_sample_h(wo, b.g.ax, b.g.ay, u1, u2);
        wi = h * (2 * dot(wo, h)) - wo;  // reflect (geometricMath.cu:197-200)
        const float sp = beckmann_D(h, b.g.ax, b.g.ay) * abs_cos(h) / (4 * abs_cos2(wo, h));
        pdf = beckmann_pdf(b.g, wo, wi);  // the pdf the next-event side evaluates (MIS pairs)
        if (!(sp > 0)) return v3(0, 0, 0);
        return beckmann_eval(b.g, b.color, b.eta, b.k, wo, wi) * (1.0f / sp);
    }
    case RT_MAT_FRESNEL_BLEND: {  // FresnelBlendMaterial.cu:143-176: its roulette always takes
                                  // this branch; the sample is h - wo, divided by pdf(wo, wi)
        pcg_float(r);  // roulette
        pcg_float(r);  // unused 2D sample
        pcg_float(r);
        const float u1 = pcg_float(r), u2 = pcg_float(r);
        const V3 h = beckmann_sample_h(wo, 0.5f, 0.5f, u1, u2);
        const V3 raw = h - wo;
        pdf = fresnel_blend_pdf(wo, raw);
        if (!(pdf > 0) || dot(raw, raw) == 0) {
            wi = v3(0, 0, 1);
            return v3(0, 0, 0);
        }
        wi = normalize(raw);  // the ray direction; the value uses the raw vector, as the reference
        return fresnel_blend_eval(wo, raw) * (1.0f / pdf);
    }
    case RT_MAT_PLASTIC: {  // PlasticUnrealMaterial.cu:61-76: Lambertian (0.7) or mirror (0.3),
                            // each returning its own value undivided; pdf() is 0
        if (pcg_float(r) < 0.7f) {
            float u1 = pcg_float(r), u2 = pcg_float(r);
            wi = cosine_hemisphere(u1, u2);
            return b.color;
        }
        delta = true;
        wi = v3(-wo.x, -wo.y, wo.z);
        return b.color;
    }
    default:  // Light (NullBSDF) and Plain: no scattering
        wi = v3(0, 0, 0);
        return v3(0, 0, 0);
    }
}

// Emitters and point lights next-event estimation draws from for a path of scene `sub`
// (all of them in a plain scene; the scene's own in a merged scene).
struct SceneLights {
    uint32_t e0, ne;  // emitters [e0, e0 + ne) of emit_tri / emit_cdf
    float etotal;     // their sum of area * luminance (the cdf's last value)
    uint32_t pl0, npl;
};
__device__ __forceinline__ SceneLights scene_lights(const RenderView &rv, uint32_t sub)
{
    if (rv.sv.subs) {
        const SubScene &ss = rv.sv.subs[min(sub, rv.sv.nsubs - 1)];
        return SceneLights{ss.e0, ss.ne, ss.etotal, ss.pl0, ss.npl};
    }
    return SceneLights{0u, rv.nemit, rv.emit_total, 0u, rv.nplights};
}

__device__ __forceinline__ float emitter_pdf(float emit_total, V3 Le, float dist2, float cosl)
{
    // p(select tri) / area = luminance(Le) / total; solid-angle conversion dist^2 / |cos|
    if (!(cosl > 0) || emit_total <= 0) return 0.f;
    return luminance(Le) / emit_total * dist2 / cosl;
}


// Host: device view of a scene for the shading kernels (uploads render data if needed).
int make_render_view(rt_scene *s, RenderView &rv);

}  // namespace rtb
