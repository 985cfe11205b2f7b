// k-nearest photon query over the implicit kd-tree and the photon density estimate,
// shared by the photon-map entry points (photon.cu) and the renderer (render.cu).
#pragma once

#include "surface.cuh"

namespace rtb {

constexpr uint32_t kKnnMaxK = 128;

// Euclidean norm as the reference evaluates it: s = 0; s += r*r per axis; sqrt
// (kdtree.h:175-176, difference kdtree.h:67-76).
__device__ __forceinline__ float ref_dist(float qx, float qy, float qz, float4 p)
{
    float dx = __fsub_rn(qx, p.x), dy = __fsub_rn(qy, p.y), dz = __fsub_rn(qz, p.z);
    float s = __fadd_rn(__fadd_rn(__fadd_rn(0.f, __fmul_rn(dx, dx)), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    return __fsqrt_rn(s);
}

// nn::KDTree::nearest_neighbors_impl (kdtree.h:111-152) without recursion: photons with
// distance < bound on the query's shape (or any, sid = -1) enter a max-heap of k; the bound
// becomes the k-th distance once k are held; the far side of a split is visited only when
// the plane is nearer than the bound. Fills hd/hi (max-heap) and returns the count.
__device__ __forceinline__ uint32_t knn_query(const float4 *__restrict__ node_pos, const int2 *__restrict__ node_aux,
                                              uint32_t n, float qx, float qy, float qz, int32_t sid, uint32_t k,
                                              float radius, float *hd, int32_t *hi)
{
    uint32_t cnt = 0;
    float rcur = radius;
    uint32_t sl[64], sr[64];
    float sd[64];
    int sp = 1;
    sl[0] = 0;
    sr[0] = n;
    sd[0] = 0.f;
    while (sp > 0) {
        sp--;
        const uint32_t l = sl[sp], r = sr[sp];
        if (!(sd[sp] < rcur) || r <= l) continue;
        const uint32_t m = (l + r) >> 1;
        const float4 p = __ldg(node_pos + m);
        const int2 aux = __ldg(node_aux + m);
        const float dist = ref_dist(qx, qy, qz, p);
        if (dist < rcur && (sid == -1 || aux.x == sid)) {
            if (cnt < k) {  // sift up
                uint32_t c = cnt++;
                while (c > 0) {
                    uint32_t par = (c - 1) >> 1;
                    if (!(hd[par] < dist)) break;
                    hd[c] = hd[par];
                    hi[c] = hi[par];
                    c = par;
                }
                hd[c] = dist;
                hi[c] = aux.y;
                if (cnt == k) rcur = hd[0];
            } else {  // replace the farthest, sift down
                uint32_t c = 0;
                for (;;) {
                    uint32_t a = 2 * c + 1, b = a + 1, big = c;
                    float bd = dist;
                    if (a < k && hd[a] > bd) {
                        big = a;
                        bd = hd[a];
                    }
                    if (b < k && hd[b] > bd) {
                        big = b;
                        bd = hd[b];
                    }
                    if (big == c) break;
                    hd[c] = hd[big];
                    hi[c] = hi[big];
                    c = big;
                }
                hd[c] = dist;
                hi[c] = aux.y;
                rcur = hd[0];
            }
        }
        if (r - l > 1) {
            const uint32_t axis = __float_as_uint(p.w);
            const float qa = axis == 0 ? qx : (axis == 1 ? qy : qz);
            const float pa = axis == 0 ? p.x : (axis == 1 ? p.y : p.z);
            const float diff = __fsub_rn(qa, pa);
            const float pd = __fsqrt_rn(__fmul_rn(diff, diff));  // norm(p - pplane) (kdtree.h:138-148)
            uint32_t nl, nr, fl, fr;
            if (qa < pa) {
                nl = l, nr = m, fl = m + 1, fr = r;
            } else {
                nl = m + 1, nr = r, fl = l, fr = m;
            }
            if (sp + 2 <= 64) {
                sl[sp] = fl, sr[sp] = fr, sd[sp] = pd, sp++;  // far side, tested again when popped
                sl[sp] = nl, sr[sp] = nr, sd[sp] = 0.f, sp++;
            }
        }
    }
    return cnt;
}

// Max-heap -> ascending distance, in place.
__device__ __forceinline__ void heap_to_sorted(float *hd, int32_t *hi, uint32_t cnt)
{
    for (uint32_t end = cnt; end > 1; end--) {
        float td = hd[0];
        int32_t ti = hi[0];
        float ld = hd[end - 1];
        int32_t li = hi[end - 1];
        uint32_t c = 0;
        const uint32_t m = end - 1;
        for (;;) {
            uint32_t a = 2 * c + 1, b = a + 1, big = c;
            float bd = ld;
            if (a < m && hd[a] > bd) {
                big = a;
                bd = hd[a];
            }
            if (b < m && hd[b] > bd) {
                big = b;
                bd = hd[b];
            }
            if (big == c) break;
            hd[c] = hd[big];
            hi[c] = hi[big];
            c = big;
        }
        hd[c] = ld;
        hi[c] = li;
        hd[end - 1] = td;
        hi[end - 1] = ti;
    }
}

// Scene::combinePhotonContributions (Scene.cu:607-635) at point p with shading normal nn and
// world outgoing direction wo_w: sum over the k nearest photons of power * f(wo, -dir)|cos|
// (SurfaceInteraction::lightScattered, SurfaceInteraction.cu:278-292) / (pi * maxDist^2).
// The reference weights each photon by |cos| although the photon density already carries the
// projected-area factor; with compat = false the estimate uses f alone (the radiance
// estimate of photon mapping).
__device__ __forceinline__ V3 photon_density(const float4 *__restrict__ node_pos, const int2 *__restrict__ node_aux,
                                             const rt_photon *__restrict__ photons, uint32_t n, const Bsdf &bs, V3 p,
                                             V3 nn, V3 wo_w, int32_t sid, uint32_t k, float radius, bool compat = true)
{
    float hd[kKnnMaxK];
    int32_t hi[kKnnMaxK];
    const uint32_t cnt = knn_query(node_pos, node_aux, n, p.x, p.y, p.z, sid, k, radius, hd, hi);
    if (cnt == 0) return v3(0, 0, 0);
    V3 t, b;
    onb(nn, t, b);
    V3 wo = v3(dot(wo_w, t), dot(wo_w, b), dot(wo_w, nn));
    V3 sum = v3(0, 0, 0);
    float maxd = 0.f;
    for (uint32_t j = 0; j < cnt; j++) {
        const rt_photon ph = photons[hi[j]];
        V3 loc = v3(ph.pos[0], ph.pos[1], ph.pos[2]);
        maxd = fmaxf(maxd, length(loc - p));
        V3 w = -v3(ph.dir[0], ph.dir[1], ph.dir[2]);
        V3 wl = v3(dot(w, t), dot(w, b), dot(w, nn));
        float pdf;
        V3 f = bsdf_eval(bs, wo, wl, pdf);
        if (!compat) {
            const float c = abs_cos(wl);
            f = c > 0 ? f * (1.0f / c) : v3(0, 0, 0);
        }
        sum = sum + v3(ph.power[0], ph.power[1], ph.power[2]) * f;
    }
    const float kernel = 1.0f / (kPi * maxd * maxd);
    return sum * kernel;
}

// nn::KDTree::nearest_neighbors with an unbounded k (kdtree.h:111-152, as
// Scene::search_nearest(p, radius, (ulong)-1, shapeId) calls it, Scene.cu:808-813): every photon
// at distance < radius on shape sid (-1: any) is passed to visit(photon index, distance).
template <class F>
__device__ __forceinline__ uint32_t radius_query(const float4 *__restrict__ node_pos, const int2 *__restrict__ node_aux,
                                                 uint32_t n, float qx, float qy, float qz, int32_t sid, float radius,
                                                 F &&visit)
{
    uint32_t cnt = 0;
    uint32_t sl[64], sr[64];
    float sd[64];
    int sp = 1;
    sl[0] = 0;
    sr[0] = n;
    sd[0] = 0.f;
    while (sp > 0) {
        sp--;
        const uint32_t l = sl[sp], r = sr[sp];
        if (!(sd[sp] < radius) || r <= l) continue;
        const uint32_t m = (l + r) >> 1;
        const float4 p = __ldg(node_pos + m);
        const int2 aux = __ldg(node_aux + m);
        const float dist = ref_dist(qx, qy, qz, p);
        if (dist < radius && (sid == -1 || aux.x == sid)) {
            visit(aux.y, dist);
            cnt++;
        }
        if (r - l > 1) {
            const uint32_t axis = __float_as_uint(p.w);
            const float qa = axis == 0 ? qx : (axis == 1 ? qy : qz);
            const float pa = axis == 0 ? p.x : (axis == 1 ? p.y : p.z);
            const float diff = __fsub_rn(qa, pa);
            const float pd = __fsqrt_rn(__fmul_rn(diff, diff));
            uint32_t nl, nr, fl, fr;
            if (qa < pa) {
                nl = l, nr = m, fl = m + 1, fr = r;
            } else {
                nl = m + 1, nr = r, fl = l, fr = m;
            }
            if (sp + 2 <= 64) {
                sl[sp] = fl, sr[sp] = fr, sd[sp] = pd, sp++;
                sl[sp] = nl, sr[sp] = nr, sd[sp] = 0.f, sp++;
            }
        }
    }
    return cnt;
}

// Radius of the subsurface gather: th_photonSubsurfaceContributions' searchRadius (Scene.cu:802).
constexpr float kSubsurfaceRadius = 0.3f;

// impPaper_dipoleDiffusionAproximation (geometricMath.cu:455-490), one channel: the dipole
// diffuse reflectance Rd at distance r with the reduced scattering coefficient (1 - g) sigma_s.
__device__ __forceinline__ float dipole_rd(float r, float ss, float sa, float g, float eta)
{
    const float rs = (1 - g) * ss;
    const float rt = rs + sa;
    const float alpha = rs / rt;
    const float tr = sqrtf(3 * sa * rt);
    const float fdr = (-1.440f / (eta * eta)) + (0.710f / eta) + 0.668f + 0.0636f * eta;
    const float A = (1 + fdr) / (1 - fdr);
    const float zr = sqrtf(3 * (1 - alpha)) / tr;
    const float zv = zr * A;
    const float dr = sqrtf(r * r + zr * zr), dv = sqrtf(r * r + zv * zv);
    const float trdr = tr * dr, trdv = tr * dv;
    const float rd = (trdr + 1) * expf(-trdr) * zr / (dr * dr * dr) + (trdv + 1) * expf(-trdv) * zv / (dv * dv * dv);
    const float c1 = zr * (tr + 1 / dr);
    return c1 * rd * (1 - fdr) * alpha;
}

// Scene::combinePhotonsSubsurface (Scene.cu:667-701) at point p (shading normal nn, direction
// to the camera wo_w) of an SSMaterial m: over the photons within `radius` on the same shape,
// sum of power * kd * diffusionTermBSSRDF (geometricMath.cu:503-522:
// Rd * (1 - F(cos_o)) * (1 - F(cos_i)) / pi) / (2 pi maxDist^2). With no photon the reference
// divides 0 by 0 (a NaN sample, which the film drops); `compat` keeps that, otherwise 0.
__device__ __forceinline__ V3 photon_subsurface(const float4 *__restrict__ node_pos,
                                                const int2 *__restrict__ node_aux,
                                                const rt_photon *__restrict__ photons, uint32_t n,
                                                const rt_material &m, V3 p, V3 nn, V3 wo_w, int32_t sid, float radius,
                                                bool compat)
{
    const float eta = m.ior, g = m.roughness[1];
    const float cos_o = dot(nn, wo_w) / (length(nn) * length(wo_w));
    const float ft_o = 1.f - fresnel_dielectric_ref(cos_o, 1.f, eta);
    V3 sum = v3(0, 0, 0);
    float maxd = 0.f;
    const uint32_t cnt = radius_query(node_pos, node_aux, n, p.x, p.y, p.z, sid, radius, [&](int32_t idx, float) {
        const rt_photon ph = photons[idx];
        const V3 loc = v3(ph.pos[0], ph.pos[1], ph.pos[2]);
        const float r = length(loc - p);
        maxd = fmaxf(maxd, r);
        const V3 pn = v3(ph.normal[0], ph.normal[1], ph.normal[2]);
        const V3 wi = -v3(ph.dir[0], ph.dir[1], ph.dir[2]);
        const float cos_i = dot(pn, wi) / (length(pn) * length(wi));
        const float s = kInvPi * (1.f - fresnel_dielectric_ref(cos_i, 1.f, eta)) * ft_o;
        const V3 rd = v3(dipole_rd(r, m.eta[0], m.extra[0], g, eta), dipole_rd(r, m.eta[1], m.extra[1], g, eta),
                         dipole_rd(r, m.eta[2], m.extra[2], g, eta));
        sum = sum + rd * s * v3(ph.power[0], ph.power[1], ph.power[2]) * v3(m.color[0], m.color[1], m.color[2]);
    });
    if (cnt == 0) return compat ? v3(NAN, NAN, NAN) : v3(0, 0, 0);
    return sum * (1.f / (2.f * kPi * maxd * maxd));
}

}  // namespace rtb
