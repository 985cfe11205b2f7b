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

// Radius of the subsurface gather: th_photonSubsurfaceContributions' searchRadius (Scene.cu:802).
constexpr float kSubsurfaceRadius = 0.3f;

// impPaper_dipoleDiffusionAproximation (geometricMath.cu:455-490), one channel: the dipole
// diffuse reflectance Rd at distance r with the reduced scattering coefficient (1 - g) sigma_s.
// The terms that do not depend on r are set up once per query (DipoleChannel); dipole_eval
// evaluates the rest per photon, the hot loop of the subsurface gather, with reciprocal square
// roots and the hardware exponential (relative error about 1e-6, against 1e-7 for the IEEE
// operations): with d = sqrt(r^2 + z^2), 1/d and 1/d^3 come from one rsqrt.
struct DipoleChannel {
    float tr, zr, zv, omf, alpha;  // sigma_tr, real and virtual source depths, 1 - Fdr, albedo
};

__device__ __forceinline__ DipoleChannel dipole_setup(float ss, float sa, float g, float eta)
{
    DipoleChannel c;
    const float rs = (1 - g) * ss;
    const float rt = rs + sa;
    c.alpha = rs / rt;
    c.tr = sqrtf(3 * sa * rt);
    const float fdr = (-1.440f / (eta * eta)) + (0.710f / eta) + 0.668f + 0.0636f * eta;
    const float A = (1 + fdr) / (1 - fdr);
    c.zr = sqrtf(3 * (1 - c.alpha)) / c.tr;
    c.zv = c.zr * A;
    c.omf = 1 - fdr;
    return c;
}

__device__ __forceinline__ float dipole_eval(const DipoleChannel &c, float r2)
{
    const float xr = r2 + c.zr * c.zr, xv = r2 + c.zv * c.zv;
    const float ir = rsqrtf(xr), iv = rsqrtf(xv);  // 1/dr, 1/dv
    const float trdr = c.tr * (xr * ir), trdv = c.tr * (xv * iv);
    const float rd = (trdr + 1) * __expf(-trdr) * c.zr * (ir * ir * ir) + (trdv + 1) * __expf(-trdv) * c.zv * (iv * iv * iv);
    const float c1 = c.zr * (c.tr + ir);
    return c1 * rd * c.omf * c.alpha;
}

// ------------------------------------------------------- warp-cooperative queries
// One warp answers one query, with its traversal stack in shared memory. Every lane of the warp
// must call these functions together. Serial per-node chains of local-memory stack and heap
// traffic are what bound the one-thread-per-query form: here a warp reads a subtree of at most
// Scan photons (a contiguous range of the implicit tree) with coalesced loads, keeps k-nearest
// candidates in a buffer that it narrows to k by a radix select, and reads the photons'
// attributes in tree order.

// Device view of a built photon map, all arrays in tree-slot order.
struct PhotonTree {
    const float4 *pos;  // xyz, split axis (uint bits)
    const int2 *aux;    // shape id, photon index
    const float4 *pw;   // power rgb, cosine of the photon's normal with its reversed direction
    const float4 *dir;  // arrival direction xyz, 0
    uint32_t n;
};

inline PhotonTree photon_tree(const rt_photon_map *m)
{
    PhotonTree t;
    t.pos = m->node_pos.as<float4>();
    t.aux = m->node_aux.as<int2>();
    t.pw = m->node_pw.as<float4>();
    t.dir = m->node_dir.as<float4>();
    t.n = (uint32_t)m->n;
    return t;
}

constexpr uint32_t kKnnScan = 64;      // scanned subtree size of a k-nearest query
constexpr uint32_t kRadiusScan = 256;  // of a fixed-radius query (no bound to tighten)
// Stack bound: a popped range is replaced by its two halves, and for n < 2^31 ranges of more
// than kKnnScan photons lie on at most 25 levels, so the stack holds at most 26 entries.
constexpr int kWarpStack = 32;
constexpr unsigned kFullMask = 0xFFFFFFFFu;

// Candidate buffer of a k-nearest query: after a selection it holds k <= kKnnMaxK, and it is
// selected again before an append could take it past kKnnBuf.
constexpr uint32_t kKnnBuf = 256;
static_assert(kKnnBuf >= 2 * kKnnMaxK, "room for k plus one batch of candidates");

struct PhotonWarpScratch {  // per warp, in shared memory
    float kd[kKnnBuf];     // candidate distances (unordered)
    uint32_t ki[kKnnBuf];  // and tree slots
    uint32_t sl[kWarpStack], sr[kWarpStack];
    float sd[kWarpStack];
};

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

__device__ __forceinline__ float warp_max(float v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFullMask, v, o));
    return v;
}

// The pruned traversal of knn_query (kdtree.h:111-152) for a warp: the same depth-first,
// near-side-first order with the same pruning (a far side is skipped when its split plane is
// not nearer than the bound), decided warp-uniformly with the stack in shared memory. A range
// of at most Scan photons is read 32 photons per load instead of node by node. bound() is the
// current search distance (warp-uniform); visit(valid, dist, shape, slot) is offered up to 32
// photons, one per lane (an internal node's photon on lane 0).
template <uint32_t Scan, class Bound, class Visit>
__device__ __forceinline__ void warp_traverse(const PhotonTree &t, float qx, float qy, float qz, PhotonWarpScratch &sm,
                                              Bound &&bound, Visit &&visit)
{
    const uint32_t lane = threadIdx.x & 31u;
    int sp = 1;
    if (lane == 0) {
        sm.sl[0] = 0;
        sm.sr[0] = t.n;
        sm.sd[0] = 0.f;
    }
    __syncwarp();
    while (sp > 0) {
        sp--;
        const uint32_t l = sm.sl[sp], r = sm.sr[sp];
        const float pd = sm.sd[sp];
        __syncwarp();  // every lane has read the entry before lane 0 reuses it
        if (!(pd < bound()) || r <= l) continue;
        if (r - l <= Scan) {
            for (uint32_t base = l; base < r; base += 64) {  // two loads in flight per lane
                const uint32_t j0 = base + lane, j1 = base + 32 + lane;
                float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
                int s0 = -1, s1 = -1;
                if (j0 < r) {
                    p0 = __ldg(t.pos + j0);
                    s0 = __ldg(&t.aux[j0].x);
                }
                if (j1 < r) {
                    p1 = __ldg(t.pos + j1);
                    s1 = __ldg(&t.aux[j1].x);
                }
                visit(j0 < r, j0 < r ? ref_dist(qx, qy, qz, p0) : INFINITY, s0, j0);
                if (base + 32 < r) visit(j1 < r, j1 < r ? ref_dist(qx, qy, qz, p1) : INFINITY, s1, j1);
            }
            continue;
        }
        const uint32_t m = (l + r) >> 1;
        const float4 p = __ldg(t.pos + m);  // one address for the warp
        visit(lane == 0, ref_dist(qx, qy, qz, p), __ldg(&t.aux[m].x), m);
        const uint32_t axis = __float_as_uint(p.w);
        const float qa = axis == 0 ? qx : (axis == 1 ? qy : qz);
        const float pa = axis == 0 ? p.x : (axis == 1 ? p.y : p.z);
        const float diff = __fsub_rn(qa, pa);
        const float pd2 = __fsqrt_rn(__fmul_rn(diff, diff));  // norm(p - pplane) (kdtree.h:138-148)
        if (sp + 2 <= kWarpStack) {  // holds for n < 2^31 (kWarpStack)
            if (lane == 0) {
                if (qa < pa) {
                    sm.sl[sp] = m + 1, sm.sr[sp] = r, sm.sd[sp] = pd2;  // far side
                    sm.sl[sp + 1] = l, sm.sr[sp + 1] = m, sm.sd[sp + 1] = 0.f;
                } else {
                    sm.sl[sp] = l, sm.sr[sp] = m, sm.sd[sp] = pd2;
                    sm.sl[sp + 1] = m + 1, sm.sr[sp + 1] = r, sm.sd[sp + 1] = 0.f;
                }
            }
            sp += 2;
        }
        __syncwarp();
    }
}

// knn_query for a warp: the same neighbour set (the k nearest photons at distance < radius on
// shape sid, -1: any), up to the order in which photons at exactly equal distances compete
// for the last place. Candidates (distance below the bound) are appended to a buffer; when it
// first holds k, and whenever it is nearly full, the k nearest are kept and the bound becomes
// the k-th distance, as the reference's heap bound does once it holds k. Leaves the neighbours' tree slots
// unordered in sm.ki; returns their count (all lanes).
__device__ __forceinline__ uint32_t warp_knn(const PhotonTree &t, float qx, float qy, float qz, int32_t sid, uint32_t k,
                                             float radius, PhotonWarpScratch &sm)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t cnt = 0, select_at = k;
    float rcur = radius;
    // keep the k nearest of cnt > k buffered: the k-th smallest distance v (bitwise search on
    // the float bits, which order like the values for distances >= 0), then the ones below it
    // and as many equal to it as fill k
    auto select = [&]() {
        uint32_t key[kKnnBuf / 32], slot[kKnnBuf / 32];
#pragma unroll
        for (uint32_t i = 0; i < kKnnBuf / 32; i++) {
            const uint32_t j = lane + 32 * i;
            key[i] = j < cnt ? __float_as_uint(sm.kd[j]) : 0xFFFFFFFFu;
            slot[i] = j < cnt ? sm.ki[j] : 0u;
        }
        // largest v with fewer than k keys below it (the k-th smallest key), or the first
        // threshold met with exactly k below it (then those k are the k nearest, no tie)
        uint32_t v = 0, less = 0;
        bool exact = false;
        for (int bit = 30; bit >= 0; bit--) {
            const uint32_t tv = v | (1u << bit);
            uint32_t c = 0;
#pragma unroll
            for (uint32_t i = 0; i < kKnnBuf / 32; i++) c += key[i] < tv;
            c = __reduce_add_sync(kFullMask, c);
            if (c == k) {
                v = tv;
                less = k;
                exact = true;
                break;
            }
            if (c < k) {
                v = tv;
                less = c;
            }
        }
        const uint32_t need = k - less;
        __syncwarp();  // every lane holds its entries before the buffer is rewritten
        uint32_t blt = 0, beq = 0;
#pragma unroll
        for (uint32_t i = 0; i < kKnnBuf / 32; i++) {
            const bool lt = key[i] < v, eq = key[i] == v;
            const unsigned mlt = __ballot_sync(kFullMask, lt), meq = __ballot_sync(kFullMask, eq);
            if (lt) {
                const uint32_t pos = blt + __popc(mlt & below);
                sm.kd[pos] = __uint_as_float(key[i]);
                sm.ki[pos] = slot[i];
            }
            if (eq && !exact) {
                const uint32_t rk = beq + __popc(meq & below);
                if (rk < need) {
                    sm.kd[less + rk] = __uint_as_float(key[i]);
                    sm.ki[less + rk] = slot[i];
                }
            }
            blt += __popc(mlt);
            beq += __popc(meq);
        }
        __syncwarp();
        cnt = k;
        // the bound: the largest kept distance (v itself unless the search stopped early)
        float mx = 0.f;
        for (uint32_t j = lane; j < k; j += 32) mx = fmaxf(mx, sm.kd[j]);
        rcur = exact ? warp_max(mx) : __uint_as_float(v);
        select_at = kKnnBuf - 32;
    };
    warp_traverse<kKnnScan>(t, qx, qy, qz, sm, [&]() { return rcur; },
                            [&](bool valid, float dist, int shape, uint32_t slot) {
                                const bool c = valid && dist < rcur && (sid == -1 || shape == sid);
                                const unsigned mask = __ballot_sync(kFullMask, c);
                                if (!mask) return;
                                if (c) {
                                    const uint32_t pos = cnt + __popc(mask & below);
                                    sm.kd[pos] = dist;
                                    sm.ki[pos] = slot;
                                }
                                cnt += __popc(mask);
                                __syncwarp();
                                if (cnt >= select_at) select();
                            });
    if (cnt > k) select();
    __syncwarp();
    return cnt;
}

// Scene::combinePhotonContributions (Scene.cu:607-635) at point p with shading normal nn and
// world outgoing direction wo_w, for a warp: sum over the k nearest photons of
// power * f(wo, -dir)|cos| (SurfaceInteraction::lightScattered, SurfaceInteraction.cu:278-292)
// / (pi * maxDist^2). The reference weights each photon by |cos| although the photon density
// already carries the projected-area factor; with compat = false the estimate uses f alone
// (the radiance estimate of photon mapping). The k terms are summed lane-parallel. Returns the
// estimate on every lane.
__device__ __forceinline__ V3 warp_photon_density(const PhotonTree &t, const Bsdf &bs, V3 p, V3 nn, V3 wo_w,
                                                  int32_t sid, uint32_t k, float radius, bool compat,
                                                  PhotonWarpScratch &sm)
{
    const uint32_t cnt = warp_knn(t, p.x, p.y, p.z, sid, k, radius, sm);
    if (cnt == 0) return v3(0, 0, 0);
    V3 tt, b;
    onb(nn, tt, b);
    const V3 wo = v3(dot(wo_w, tt), dot(wo_w, b), dot(wo_w, nn));
    V3 sum = v3(0, 0, 0);
    float maxd = 0.f;
    for (uint32_t j = threadIdx.x & 31u; j < cnt; j += 32) {
        const uint32_t s = sm.ki[j];
        const float4 pp = __ldg(t.pos + s), pw = __ldg(t.pw + s), pd = __ldg(t.dir + s);
        maxd = fmaxf(maxd, length(v3(pp.x, pp.y, pp.z) - p));
        const V3 w = -v3(pd.x, pd.y, pd.z);
        const V3 wl = v3(dot(w, tt), dot(w, b), dot(w, nn));
        float pdf;
        V3 f = bsdf_eval(bs, wo, wl, pdf);
        if (!compat) {
            const float c = abs_cos(wl);
            f = c > 0 ? f * (1.0f / c) : v3(0, 0, 0);
        }
        sum = sum + v3(pw.x, pw.y, pw.z) * f;
    }
    sum = v3(warp_sum(sum.x), warp_sum(sum.y), warp_sum(sum.z));
    maxd = warp_max(maxd);
    return sum * (1.0f / (kPi * maxd * maxd));
}

// Scene::combinePhotonsSubsurface (Scene.cu:667-701) at point p (shading normal nn, direction
// to the camera wo_w) of an SSMaterial m with diffuse colour kd (m's kd, times its texel at
// the point when it has a texture: SSMaterial::getBSSDFparameters, SSMaterial.cu:245-263), for a warp. Over the photons within `radius` on the
// same shape (nn::KDTree::nearest_neighbors with an unbounded k, as
// Scene::search_nearest(p, radius, (ulong)-1, shapeId) calls it, Scene.cu:808-813): sum of
// power * kd * diffusionTermBSSRDF (geometricMath.cu:503-522:
// Rd * (1 - F(cos_o)) * (1 - F(cos_i)) / pi) / (2 pi maxDist^2). With no photon the reference
// divides 0 by 0 (a NaN sample, which the film drops); `compat` keeps that, otherwise 0. The
// terms are summed lane-parallel. Returns the estimate on every lane.
__device__ __forceinline__ V3 warp_photon_subsurface(const PhotonTree &t, const rt_material &m, V3 kd, V3 p, V3 nn,
                                                     V3 wo_w, int32_t sid, float radius, bool compat,
                                                     PhotonWarpScratch &sm)
{
    const float eta = m.ior, g = m.roughness[1];
    const float cos_o = dot(nn, wo_w) / (length(nn) * length(wo_w));
    const float ft_o = 1.f - fresnel_dielectric_ref(cos_o, 1.f, eta);
    const DipoleChannel d0 = dipole_setup(m.eta[0], m.extra[0], g, eta), d1 = dipole_setup(m.eta[1], m.extra[1], g, eta),
                        d2 = dipole_setup(m.eta[2], m.extra[2], g, eta);
    V3 sum = v3(0, 0, 0);
    float maxd = 0.f;
    uint32_t cnt = 0;
    auto add = [&](uint32_t s, float r) {  // r: the photon's distance, as the search measured it
        const float4 pw = __ldg(t.pw + s);
        maxd = fmaxf(maxd, r);
        const float sc = kInvPi * (1.f - fresnel_dielectric_ref(pw.w, 1.f, eta)) * ft_o;
        const float r2 = r * r;
        const V3 rd = v3(dipole_eval(d0, r2), dipole_eval(d1, r2), dipole_eval(d2, r2));
        sum = sum + rd * sc * v3(pw.x, pw.y, pw.z) * kd;
    };
    warp_traverse<kRadiusScan>(t, p.x, p.y, p.z, sm, [&]() { return radius; },
                               [&](bool valid, float dist, int shape, uint32_t s) {
                                   const bool ok = valid && dist < radius && (sid == -1 || shape == sid);
                                   cnt += __popc(__ballot_sync(kFullMask, ok));
                                   if (ok) add(s, dist);
                               });
    if (cnt == 0) return compat ? v3(NAN, NAN, NAN) : v3(0, 0, 0);
    sum = v3(warp_sum(sum.x), warp_sum(sum.y), warp_sum(sum.z));
    maxd = warp_max(maxd);
    return sum * (1.f / (2.f * kPi * maxd * maxd));
}

}  // namespace rtb
