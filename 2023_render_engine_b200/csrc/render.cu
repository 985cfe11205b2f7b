// Wavefront path tracer (sm_100a): the reference's PathTracerIntegrator bounce loop
// (integration/pathTracing.cu:284-414, PathTracerIntegrator.cu:26-210) as queues of
// independent paths.
//
// One wave = one bounce of every path in flight:
//   extend  - closest hit of the wave's rays (BVH8 traversal, trace.cu)
//   shade   - per path: emission, next-event estimation (point lights as the reference,
//             plus area lights with MIS when enabled), BSDF sampling, Russian roulette;
//             continuing paths are appended to the next wave's queue, finished paths to
//             the retire list, and a freed slot immediately starts the next camera sample
//             (path regeneration)
//   shadow  - any-hit test of the shadow rays; unoccluded contributions are added to the
//             path they belong to
//   retire  - finished paths add their radiance to the film (NaN/Inf samples dropped)
// Path state moves with the queue (double-buffered SoA), so every stage reads and writes
// its arrays with coalesced 16-byte accesses; queue appends are warp-aggregated.
//
// Guided mode (RT_RENDER_GUIDE) adds an inference kernel between extend and shade: the
// guide network maps each hit to a vMF mixture, and shade samples it or the BSDF (one-sample
// MIS, density alpha * guide + (1 - alpha) * bsdf). With training on, every guided vertex
// appends a record; radiance found later on the path (emission hits, unoccluded shadow rays)
// is added to the path's newest record, and retire turns those into suffix sums, i.e. the
// radiance each vertex's sampled direction carried back.
#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "guide.cuh"
#include "photon_query.cuh"

namespace rtb {

namespace {

constexpr int kB = 128;

// flags in st2.w
constexpr uint32_t kDepthMask = 0xFFu;
constexpr uint32_t kCameraRay = 0x100u;
constexpr uint32_t kLastSpecular = 0x200u;

constexpr uint32_t kRetireTarget = 0x80000000u;
constexpr uint32_t kRecBits = kRecNone << kRecShift;  // newest guide record of the path

struct Buffers {
    rt_ray *rays[2];
    float4 *st0[2];  // beta.xyz, pdf of the last BSDF sample
    float4 *st1[2];  // L.xyz, pixel index bits
    uint4 *st2[2];   // rng state lo/hi, sample index, flags
    rt_hit *hits;
    rt_ray *srays;
    float4 *scontrib;  // rgb, target index bits (kRetireTarget: retire list)
    float4 *retire;    // L.xyz, pixel index bits
    float4 *gather;    // photon-map gather requests, 4 float4 each: p+shape, n+material, wo+target, beta
    const uint32_t *perm;  // shading order of the wave's queue slots (material sort), or null
    uint32_t cap, scap, gcap;
    // counters (uint32): [0],[1] queue sizes of buffers 0/1, [2] shadow count, [3] retire count,
    // [4] status, [5] shadow-kernel work counter, [6] gather requests, [7] gather-kernel work
    // counter; u64 at [8]: next sample,
    // [10] extension rays, [12] shadow rays, [14] gathers; [16] guide wait timed out, [18] waves
    // of the device-side loop, [19] wave cap reached
    uint32_t *cnt;
};

struct GuideView {
    const GuideParams *params;  // per queue slot; null while the guide is untrained (BSDF sampling)
    GuideRecord *recs;
    uint32_t *rcnt;        // [0] records, [1] nonzero-weight records
    uint32_t *nz;          // records with nonzero weight
    uint32_t *retire_rec;  // newest record of each retiring path
    uint32_t rec_cap;
    uint32_t max_depth;  // vertices at this path depth or deeper sample the BSDF only
    int enabled, train;
};

// vertices that sample with the guide: diffuse and rough-conductor BSDFs, seen from the side
// their BSDF sampler covers
__device__ __forceinline__ bool guide_vertex(const Bsdf &b, float wo_z)
{
    return wo_z > 0.f &&
           (b.type == RT_MAT_LAMBERTIAN || (b.type == RT_MAT_TROWBRIDGE && fmaxf(b.g.ax, b.g.ay) >= 1e-3f));
}

// density of bsdf_sample's direction at wi (shading space), for the guide vertices
__device__ __forceinline__ float bsdf_sampling_pdf(const Bsdf &b, V3 wo, V3 wi)
{
    if (b.type == RT_MAT_LAMBERTIAN) return wi.z > 0.f ? wi.z * kInvPi : 0.f;
    if (b.type == RT_MAT_TROWBRIDGE) return ggx_pdf(b.g, normalize(wo), wi);
    return 0.f;
}

__device__ __forceinline__ unsigned long long *cnt64(uint32_t *c, int i)
{
    return reinterpret_cast<unsigned long long *>(c + i);
}

// Camera sample g of this call -> primary path in slot q of buffer b.
// Sampler::getCameraSample (Sampler.cu:165-180) + ProjectiveCamera::generateRay
// (ProjectiveCamera.cu:71-104).
__device__ void start_path(const RenderView &rv, const Buffers &bf, int b, uint32_t q, uint64_t g)
{
    const uint32_t vi = view_of_sample(rv, g);
    const rt_view &vw = rv.views[vi];
    const rt_camera &cam = vw.camera;
    g -= rv.view_sample0[vi];
    const uint32_t W = cam.width, H = cam.height;
    const uint32_t pix = (uint32_t)(g / vw.spp);
    const uint32_t j = vw.sample_offset + (uint32_t)(g % vw.spp);
    const uint32_t px = pix % W, py = pix / W;
    Pcg r = pcg_init(pix, j, vw.seed);
    float fx = fminf(fmaxf((float)px + pcg_float(r), 0.f), (float)W);
    float fy = fminf(fmaxf((float)py + pcg_float(r), 0.f), (float)H);
    float l1 = pcg_float(r), l2 = pcg_float(r);
    V3 pc = xform_point(cam.raster_to_camera, v3(fx, fy, 0.f));
    V3 oc = v3(0, 0, 0), dc = normalize(pc);
    if (cam.lens_radius > 0) {
        float lx, ly;
        concentric_disk(l1, l2, lx, ly);
        lx *= cam.lens_radius;
        ly *= cam.lens_radius;
        float ft = cam.focal_distance / pc.z;
        V3 pf = pc * ft;
        oc = v3(lx, ly, 0);
        dc = normalize(pf - oc);
    }
    V3 o = xform_point(cam.camera_to_world, oc);
    V3 d = normalize(xform_vec(cam.camera_to_world, dc));
    rt_ray ray;
    ray.ox = o.x;
    ray.oy = o.y;
    ray.oz = o.z;
    ray.tmax = INFINITY;
    ray.dx = d.x;
    ray.dy = d.y;
    ray.dz = d.z;
    ray.flags = 0;
    reinterpret_cast<float4 *>(bf.rays[b])[2 * q] = make_float4(ray.ox, ray.oy, ray.oz, ray.tmax);
    // the last word carries the view's scene (merged scenes; 0 otherwise)
    reinterpret_cast<float4 *>(bf.rays[b])[2 * q + 1] = make_float4(ray.dx, ray.dy, ray.dz, __uint_as_float(vw.scene));
    bf.st0[b][q] = make_float4(1.f, 1.f, 1.f, 0.f);
    bf.st1[b][q] = make_float4(0.f, 0.f, 0.f, __uint_as_float(rv.view_pixel0[vi] + pix));
    bf.st2[b][q] = make_uint4((uint32_t)r.state, (uint32_t)(r.state >> 32), j, kCameraRay | kRecBits);
}

// Takes the next camera sample (if any) and appends it to buffer b.
// Sample indices are handed out with one atomic per group of converged lanes.
__device__ __forceinline__ void regenerate(const RenderView &rv, const Buffers &bf, int b)
{
    cg::coalesced_group grp = cg::coalesced_threads();
    unsigned long long base = 0;
    if (grp.thread_rank() == 0) base = atomicAdd(cnt64(bf.cnt, 8), (unsigned long long)grp.size());
    const unsigned long long g = grp.shfl(base, 0) + grp.thread_rank();
    if (g >= rv.total) return;
    uint32_t q = append(bf.cnt + b);
    start_path(rv, bf, b, q, g);
}

__global__ void __launch_bounds__(kB) k_start(RenderView rv, Buffers bf)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bf.cap) return;
    regenerate(rv, bf, 0);
}

// skip_transparent: the reference's checkShadow semantics (Scene::isVisible ->
// Triangle::intersects(checkShadow), Triangle.cu:439-440): transparent materials cast no
// shadow. Used for point lights in compat mode; area-light samples must be blocked by
// glass so that their MIS pairing with BSDF-sampled emitter hits stays unbiased.
// rec: the guide record the contribution also belongs to (kRecNone: none).
// The shadow ray's last word: bit 0 skip_transparent, bits 1..22 the guide record, bits 24..31
// the path's scene (merged scenes).
constexpr uint32_t kShadowSceneShift = 24;
__device__ __forceinline__ void push_shadow(const Buffers &bf, V3 o, V3 d, float tmax, V3 contrib, uint32_t target,
                                            bool skip_transparent, uint32_t sub, uint32_t rec = kRecNone)
{
    uint32_t i = append(bf.cnt + 2);
    if (i >= bf.scap) return;
    reinterpret_cast<float4 *>(bf.srays)[2 * i] = make_float4(o.x, o.y, o.z, tmax);
    reinterpret_cast<float4 *>(bf.srays)[2 * i + 1] = make_float4(
        d.x, d.y, d.z, __uint_as_float((sub << kShadowSceneShift) | (rec << 1) | (skip_transparent ? 1u : 0u)));
    bf.scontrib[i] = make_float4(contrib.x, contrib.y, contrib.z, __uint_as_float(target));
}

constexpr uint32_t kGatherDensity = 0, kGatherSubsurface = 1;

// Queues a photon-map gather at surface sf, weighted by `weight`, for the path whose radiance
// lives at `target` (kRetireTarget: the retire list). Five float4: point + shape, normal +
// material, direction to the previous vertex + target, weight + (kind | guide record << 1),
// the material's kd at the point (its texture applied).
// rec: the guide record the estimate also belongs to (kRecNone: none).
constexpr int kGatherWords = 5;
__device__ __forceinline__ void push_gather(const Buffers &bf, const Surface &sf, V3 wo_w, V3 weight, uint32_t target,
                                            uint32_t kind, uint32_t rec, V3 kd)
{
    const uint32_t gi = append(bf.cnt + 6);
    if (gi >= bf.gcap) return;
    float4 *g = bf.gather + (uint64_t)kGatherWords * gi;
    g[0] = make_float4(sf.p.x, sf.p.y, sf.p.z, __int_as_float(sf.shape));
    g[1] = make_float4(sf.n.x, sf.n.y, sf.n.z, __uint_as_float(sf.mat));
    g[2] = make_float4(wo_w.x, wo_w.y, wo_w.z, __uint_as_float(target));
    g[3] = make_float4(weight.x, weight.y, weight.z, __uint_as_float(kind | (rec << 1)));
    g[4] = make_float4(kd.x, kd.y, kd.z, 0.f);
}

struct PhotonView {
    PhotonTree tree;
    uint32_t k;
    float radius;
};

// Material sort: the shading order of a wave. Each block takes chunks of 2^log2 queue slots
// and orders each by the kind of surface its ray hit (a miss first, then rt_material_type), by
// a stable counting sort in shared memory; k_shade's thread i then shades slot perm[i]. Lanes of a warp
// then mostly run the same BSDF code, while the chunk keeps the state reads of a warp within a
// few kilobytes. The chunk size is the sort granularity (rt_render_set_sort).
constexpr int kSortBlock = 256;
constexpr int kSortKeys = 16;  // 0: miss, 1 + rt_material_type
constexpr uint32_t kSortMaxLog2 = 13;
__device__ __forceinline__ uint32_t shade_key(const RenderView &rv, const Buffers &bf, uint32_t q)
{
    const int32_t prim = __float_as_int(__ldg(reinterpret_cast<const float *>(bf.hits) + 4 * (uint64_t)q + 1));
    if (prim < 0) return 0;
    uint32_t mat;
    if (prim & RT_PRIM_SHAPE)
        mat = rv.sv.spheres[prim & ~RT_PRIM_SHAPE].material;
    else
        mat = __ldg(rv.tri_mat + prim);
    const uint32_t type = (uint32_t)rv.mats[min(mat, rv.nmats - 1)].type;
    return min(1u + type, (uint32_t)kSortKeys - 1u);
}

__global__ void __launch_bounds__(kSortBlock) k_material_sort(RenderView rv, Buffers bf, int cur, uint32_t *perm,
                                                               uint32_t log2)
{
    __shared__ uint32_t count[kSortKeys], start[kSortKeys];
    __shared__ uint8_t key[1u << kSortMaxLog2];
    __shared__ uint32_t wcount[kSortBlock / 32][kSortKeys];
    const uint32_t n = min(bf.cnt[cur], bf.cap);
    // chunks in a grid-stride loop over the resident blocks (c0 is the same for the whole block)
    for (uint32_t c0 = blockIdx.x << log2; c0 < n; c0 += gridDim.x << log2) {
        const uint32_t len = min(1u << log2, n - c0);
        if (threadIdx.x < kSortKeys) count[threadIdx.x] = 0;
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < len; j += kSortBlock) {
            const uint32_t k = shade_key(rv, bf, c0 + j);
            key[j] = (uint8_t)k;
            atomicAdd(&count[k], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int k = 0; k < kSortKeys; k++) {
                start[k] = acc;
                acc += count[k];
            }
        }
        __syncthreads();
        // stable scatter: within a key the slots keep their queue order, so that a warp of k_shade
        // reads nearly consecutive slots of the dominant material (render 2213 against 2190-2205
        // Mrays/s with the atomic, unordered scatter). Per 256-entry step, a slot's rank among
        // the same key in its warp (match + popc), then the warps' counts per key scanned in
        // warp order on top of the key's running start.
        const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
        for (uint32_t j0 = 0; j0 < len; j0 += kSortBlock) {
            const uint32_t j = j0 + threadIdx.x;
            const uint32_t k = j < len ? key[j] : (uint32_t)kSortKeys;  // kSortKeys: no entry
            if (threadIdx.x < (kSortBlock / 32) * kSortKeys) wcount[threadIdx.x / kSortKeys][threadIdx.x % kSortKeys] = 0;
            __syncthreads();
            const unsigned same = __match_any_sync(0xFFFFFFFFu, k);
            const unsigned below = same & ((1u << lane) - 1u);
            if (below == 0 && k < (uint32_t)kSortKeys) wcount[warp][k] = __popc(same);
            __syncthreads();
            if (threadIdx.x < kSortKeys) {
                uint32_t acc = start[threadIdx.x];
                for (int w = 0; w < kSortBlock / 32; w++) {
                    const uint32_t c = wcount[w][threadIdx.x];
                    wcount[w][threadIdx.x] = acc;
                    acc += c;
                }
                start[threadIdx.x] = acc;
            }
            __syncthreads();
            if (k < (uint32_t)kSortKeys) perm[c0 + wcount[warp][k] + __popc(below)] = c0 + j;
            __syncthreads();  // wcount, and after the last step count, start and key, are reused
        }
    }
}

// End of one 4-wave group of the device-side wave loop: counts the waves and sets the loop's
// condition to 0 once every queue has drained and every camera sample has started (what the
// host loop checks after each group), when the guide's tensor-core wait timed out, or at the
// wave cap (cnt[19] = 1 then). cnt[18] counts the waves.
__global__ void k_wave_check(uint32_t *cnt, uint64_t total, uint32_t max_waves, cudaGraphConditionalHandle loop)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t waves = cnt[18] + 4;
    cnt[18] = waves;
    const unsigned long long next = *reinterpret_cast<const unsigned long long *>(cnt + 8);
    const bool done = cnt[0] == 0 && next >= total;
    const bool capped = !done && waves >= max_waves;
    if (capped) cnt[19] = 1;
    cudaGraphSetConditional(loop, (done || capped || cnt[16] != 0) ? 0u : 1u);
}

// Resident blocks per SM k_shade is compiled for: more resident warps hide its scattered
// loads better than the spills they cost. BVH-stress render, Mrays/s: 1465 / 1494 / 1507 for
// 4 (127 registers, no bound) / 5 (96) / 6 (80) with the binned-SAH tree; 1559 / 1583 / 1588
// for 6 / 7 (72) / 8 (64) with the PLOC tree.
#ifndef RTB_SHADE_MIN_BLOCKS
#define RTB_SHADE_MIN_BLOCKS 8
#endif
// One thread per queue position i of the wave (the slot perm[i] when the queue is sorted), on a
// grid of the queue's capacity. A grid-stride loop over the resident blocks instead nearly
// doubles the spills at the 64-register bound (708 -> 1300 bytes of spill stores) and was 13%
// slower on the BVH-stress render (1806 -> 1578 Mrays/s at 2^22 paths).
__global__ void __launch_bounds__(kB, RTB_SHADE_MIN_BLOCKS) k_shade(RenderView rv, Buffers bf, int cur, GuideView gv)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = min(bf.cnt[cur], bf.cap);
    if (i == 0) atomicAdd(cnt64(bf.cnt, 10), (unsigned long long)n);  // extension rays of this wave
    if (i >= n) return;
    // the queue slot this thread shades. Forwarding the slot's hit, triangle record position and
    // material through the sort (32 B per path, read here in one coalesced load, so that the
    // record and material loads start one hop earlier) measured slower: 2189 against 2209 Mrays/s
    // on the BVH-stress render (more spills here, more traffic in the sort)
    const uint32_t q = bf.perm ? __ldg(bf.perm + i) : i;
    const int nxt = cur ^ 1;
    const bool compat = (rv.flags & RT_RENDER_COMPAT) != 0;
    const uint32_t sub = rv.sv.subs ? __float_as_uint(__ldg(reinterpret_cast<const float *>(bf.rays[cur]) + 8 * q + 7)) : 0u;
    const SceneLights lights = scene_lights(rv, sub);
    const bool nee_area = (rv.flags & RT_RENDER_NEE_AREA) != 0 && lights.ne > 0;
    const bool photon_mode = (rv.flags & RT_RENDER_PHOTON_MAP) != 0;
    const bool hybrid = (rv.flags & RT_RENDER_HYBRID) != 0;
    const bool subsurface = (rv.flags & RT_RENDER_SUBSURFACE) != 0;
    float4 r0 = reinterpret_cast<const float4 *>(bf.rays[cur])[2 * q];
    float4 r1 = reinterpret_cast<const float4 *>(bf.rays[cur])[2 * q + 1];
    float4 s0 = bf.st0[cur][q], s1 = bf.st1[cur][q];
    uint4 s2 = bf.st2[cur][q];
    float4 hv = reinterpret_cast<const float4 *>(bf.hits)[q];
    rt_hit h{hv.x, __float_as_int(hv.y), hv.z, hv.w};
    V3 o = v3(r0.x, r0.y, r0.z), d = v3(r1.x, r1.y, r1.z);
    V3 beta = v3(s0.x, s0.y, s0.z), L = v3(s1.x, s1.y, s1.z);
    const float last_pdf = s0.w;
    const uint32_t pix = __float_as_uint(s1.w);
    uint32_t flags = s2.w;
    const uint32_t depth = flags & kDepthMask;
    uint32_t rec = (flags >> kRecShift) & kRecNone;  // newest guide record of this path
    Pcg rng;
    rng.state = ((uint64_t)s2.y << 32) | s2.x;
    const rt_view &vw = rv.views[view_of_pixel(rv, pix)];
    rng.inc = ((((uint64_t)s2.z << 32) | vw.seed) << 1u) | 1u;

    bool finished = h.prim < 0;  // missed: no environment light (Scene::getEnvironmentLight = 0)
    uint32_t target = 0;
    bool cont = false;
    V3 next_o, next_d;
    float next_pdf = 0.f;
    uint32_t next_flags = 0;
    if (!finished) {
        Surface sf = surface_at(rv, h, o, d, compat);
        const rt_material &m = rv.mats[min(sf.mat, rv.nmats - 1)];
        Bsdf bs = load_bsdf(m);
        V3 t, bvec;
        onb(sf.n, t, bvec);
        V3 wo_w = -d;
        V3 wo = v3(dot(wo_w, t), dot(wo_w, bvec), dot(wo_w, sf.n));
        // the reference decides these from the material's own kd, before any texture
        const bool scattering = is_scattering(bs);
        const bool specular = is_specular(bs);
        const bool guide_ok = guide_vertex(bs, wo.z);
        if (m.texture) {
            const float2 uv = surface_uv(rv, h, sf);
            texture_bsdf(bs, tex_color(rv, m.texture - 1u, uv.x, uv.y));
        }
        // where this path's radiance will live after this bounce: decided below, but shadow
        // rays need the target now, so reserve it first.
        // BSDF sample first (its outcome decides continue/retire), NEE uses beta before update.
        V3 wi_l;
        float pdf_b;
        bool delta;
        V3 beta_in = beta;
        // emission of the hit surface (pathTracing.cu:49-50)
        V3 Le = v3(0, 0, 0);
        if (bs.type == RT_MAT_LIGHT) {
            Le = bs.color * m.intensity;
        } else if (bs.type == RT_MAT_PLAIN && (flags & kCameraRay)) {
            Le = bs.color;  // PlainMaterial::getEmittedRadiance on camera rays
        } else if (bs.type == RT_MAT_FRESNEL_BLEND) {
            Le = v3(m.extra[0], m.extra[1], m.extra[2]);  // FresnelBlendMaterial::getEmittedRadiance: ke
        }
        if (!is_black(Le)) {
            float w = 1.f;
            if (nee_area && bs.type == RT_MAT_LIGHT && depth > 0 && !(flags & kLastSpecular) && sf.emissive_tri) {
                float pl = emitter_pdf(lights.etotal, Le, h.t * h.t, sf.area_cos);
                w = (last_pdf * last_pdf) / (last_pdf * last_pdf + pl * pl);
            }
            L = L + beta_in * Le * w;
            // the guide is not trained on emitters that next-event estimation samples: with
            // area NEE on, the direct light is NEE's job and the guide learns the rest
            if (gv.train && rec != kRecNone && !(nee_area && bs.type == RT_MAT_LIGHT && sf.emissive_tri)) {
                float4 &e = gv.recs[rec].e;
                e.x += beta_in.x * Le.x * w;
                e.y += beta_in.y * Le.y * w;
                e.z += beta_in.z * Le.z * w;
            }
        }
        const bool guided = gv.enabled && depth < gv.max_depth && guide_ok;
        const uint32_t rec_in = rec;  // this vertex's NEE belongs to the previous record
        float alpha = 0.f;
        const GuideParams *gp = nullptr;
        if (guided && gv.params) {
            gp = gv.params + q;
            alpha = gp->alpha;
        }
        V3 f, wi_w;
        if (guided) {
            // one-sample MIS between the guide's vMF mixture and the BSDF
            const float usel = pcg_float(rng);
            if (usel < alpha) {
                const float u1 = pcg_float(rng), u2 = pcg_float(rng);
                wi_w = guide_sample(*gp, usel / alpha, u1, u2);
                wi_l = v3(dot(wi_w, t), dot(wi_w, bvec), dot(wi_w, sf.n));
            } else {
                (void)bsdf_sample(bs, wo, rng, compat, wi_l, pdf_b, delta);
                wi_w = t * wi_l.x + bvec * wi_l.y + sf.n * wi_l.z;
            }
            float pe;
            V3 fc = bsdf_eval(bs, wo, wi_l, pe);
            pdf_b = bsdf_sampling_pdf(bs, wo, wi_l);
            const float pmix = (alpha > 0.f ? alpha * guide_pdf(*gp, wi_w) : 0.f) + (1.f - alpha) * pdf_b;
            f = (pdf_b > 0.f && pmix > 0.f) ? fc * (1.f / pmix) : v3(0, 0, 0);
            delta = false;
            if (gv.train && !is_black(f)) {
                const uint32_t ri = append(gv.rcnt);
                if (ri < gv.rec_cap) {
                    GuideRecord r;
                    r.a = make_float4(sf.p.x, sf.p.y, sf.p.z, sf.n.x);
                    r.b = make_float4(sf.n.y, sf.n.z, wo_w.x, wo_w.y);
                    r.c = make_float4(wo_w.z, wi_w.x, wi_w.y, wi_w.z);
                    r.d = make_float4(pdf_b, beta_in.x, beta_in.y, beta_in.z);
                    r.e = make_float4(0.f, 0.f, 0.f, __uint_as_float(rec));
                    gv.recs[ri] = r;
                    rec = ri;
                }
            }
            pdf_b = pmix;  // the density MIS pairs with area-light sampling
        } else {
            f = bsdf_sample(bs, wo, rng, compat, wi_l, pdf_b, delta);
            wi_w = t * wi_l.x + bvec * wi_l.y + sf.n * wi_l.z;
        }
        beta = beta * f;
        finished = is_black(f);
        if (photon_mode && scattering) {
            // RENDER_MODE PHOTON_MAPPING: the density estimate at this hit ends the path
            // (Scene::getPhotonContributions, Scene.cu:822-840; finishStep, pathTracing.cu:85-89)
            finished = true;
            const uint32_t rt = kRetireTarget | append(bf.cnt + 3);
            push_gather(bf, sf, wo_w, beta_in, rt, kGatherDensity, rec_in, bs.color);
            if (subsurface && bs.type == RT_MAT_SUBSURFACE && (flags & kCameraRay))
                push_gather(bf, sf, wo_w, beta_in, rt, kGatherSubsurface, rec_in, bs.color);
            bf.retire[rt & ~kRetireTarget] = make_float4(L.x, L.y, L.z, __uint_as_float(pix));
            regenerate(rv, bf, nxt);
            return;
        }
        // Russian roulette (pathTracing.cu:91-102) on the reference's brightness (luminance) in
        // compat mode; on the largest component otherwise, so that no channel of a surviving
        // path's throughput grows past 1 (luminance lets a saturated red path grow 4.7x)
        if (!finished && scattering && depth > vw.rr_depth) {
            float qrr = fmaxf(0.05f, 1.f - (compat ? luminance(beta) : fmaxf(beta.x, fmaxf(beta.y, beta.z))));
            if (pcg_float(rng) < qrr)
                finished = true;
            else
                beta = beta * (1.f / (1.f - qrr));
        }
        if (!finished && depth + 1 >= vw.max_depth) finished = true;  // loop bound (pathTracing.cu:296)
        // reserve the path's slot for the shadow contributions
        if (!finished) {
            uint32_t qn = append(bf.cnt + nxt);
            target = qn;
            cont = true;
            next_o = spawn_origin(sf.p, sf.n, sf.perr, wi_w);
            next_d = wi_w;
            next_pdf = delta ? 0.f : pdf_b;
            next_flags = (depth + 1) | (delta ? kLastSpecular : 0u) |
                         (((flags & kCameraRay) && specular) ? kCameraRay : 0u) | (rec << kRecShift);
        } else {
            target = kRetireTarget | append(bf.cnt + 3);
        }
        // next-event estimation with beta before this bounce (pathTracing.cu:173-205). The
        // direct-light term of a vertex (Scene::sampleDirectLight, Scene.cu:914-969) also holds
        // the subsurface estimate at camera-ray hits and, in hybrid mode, the photon density,
        // with the sum halved.
        const float dscale = hybrid ? 0.5f : 1.0f;
        if (scattering) {
            if (subsurface && bs.type == RT_MAT_SUBSURFACE && (flags & kCameraRay))
                push_gather(bf, sf, wo_w, beta_in * dscale, target, kGatherSubsurface, rec_in, bs.color);
            if (hybrid) push_gather(bf, sf, wo_w, beta_in * dscale, target, kGatherDensity, rec_in, bs.color);
            for (uint32_t li = lights.pl0; li < lights.pl0 + lights.npl; li++) {  // Scene::estimateAllDirectLights
                float4 lp = rv.plights[2 * li], li4 = rv.plights[2 * li + 1];
                V3 tol = v3(lp.x, lp.y, lp.z) - sf.p;
                float dist2 = dot(tol, tol), dist = sqrtf(dist2);
                V3 wl = tol * (1.0f / dist);
                float ul1 = pcg_float(rng), ul2 = pcg_float(rng);
                (void)ul1;
                (void)ul2;
                if (!(dot(wl, sf.n) > 0)) continue;  // isOrientedTo
                V3 wls = v3(dot(wl, t), dot(wl, bvec), dot(wl, sf.n));
                float pb;
                V3 fl = bsdf_eval(bs, wo, wls, pb);
                V3 Li = v3(li4.x, li4.y, li4.z) * (1.0f / dist2);
                if (is_black(fl) || is_black(Li)) continue;
                float w = compat ? 1.0f / (1.0f + pb * pb) : 1.0f;  // powerHeuristic(1,1,1,pdf), Scene.cu:331
                V3 c = beta_in * fl * Li * (w * dscale);
                V3 so = spawn_origin(sf.p, sf.n, sf.perr, wl);
                push_shadow(bf, so, wl, dist, c, target, compat, sub, rec_in);
            }
            if (nee_area) {
                float u0 = pcg_float(rng), u1 = pcg_float(rng), u2 = pcg_float(rng);
                // pick an emitter by area * luminance
                float x = u0 * lights.etotal;
                uint32_t lo = lights.e0, hi = lights.e0 + lights.ne - 1;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (rv.emit_cdf[mid] <= x)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                uint32_t etri = rv.emit_tri[lo];
                const TriRecord er = rv.sv.tris[rv.sv.leafpos[etri]];
                V3 e0 = v3(er.v0.x, er.v0.y, er.v0.z), e1 = v3(er.v1.x, er.v1.y, er.v1.z),
                   e2 = v3(er.v2.x, er.v2.y, er.v2.z);
                float su = sqrtf(u1);
                float c0 = 1 - su, c1 = u2 * su;
                V3 xl = e0 * c0 + e1 * c1 + e2 * (1 - c0 - c1);
                V3 nl = normalize(cross(e1 - e0, e2 - e0));
                V3 tol = xl - sf.p;
                float dist2 = dot(tol, tol), dist = sqrtf(dist2);
                V3 wl = tol * (1.0f / dist);
                float cosl = fabsf(dot(nl, wl));
                const rt_material &em = rv.mats[min(rv.tri_mat[etri], rv.nmats - 1)];
                V3 Lel = v3(em.color[0], em.color[1], em.color[2]) * em.intensity;
                float pl = emitter_pdf(lights.etotal, Lel, dist2, cosl);
                if (pl > 0 && dot(wl, sf.n) > 0) {
                    V3 wls = v3(dot(wl, t), dot(wl, bvec), dot(wl, sf.n));
                    float pb;
                    V3 fl = bsdf_eval(bs, wo, wls, pb);
                    if (guided)
                        pb = (alpha > 0.f ? alpha * guide_pdf(*gp, wl) : 0.f) +
                             (1.f - alpha) * bsdf_sampling_pdf(bs, wo, wls);
                    if (!is_black(fl)) {
                        float w = (pl * pl) / (pl * pl + pb * pb);
                        V3 c = beta_in * fl * Lel * (w * dscale / pl);
                        V3 so = spawn_origin(sf.p, sf.n, sf.perr, wl);
                        push_shadow(bf, so, wl, dist * (1.0f - 1e-4f), c, target, false, sub, rec_in);
                    }
                }
            }
        }
    } else {
        target = kRetireTarget | append(bf.cnt + 3);
    }
    if (cont) {
        const uint32_t qn = target;
        reinterpret_cast<float4 *>(bf.rays[nxt])[2 * qn] = make_float4(next_o.x, next_o.y, next_o.z, INFINITY);
        reinterpret_cast<float4 *>(bf.rays[nxt])[2 * qn + 1] =
            make_float4(next_d.x, next_d.y, next_d.z, __uint_as_float(sub));
        bf.st0[nxt][qn] = make_float4(beta.x, beta.y, beta.z, next_pdf);
        bf.st1[nxt][qn] = make_float4(L.x, L.y, L.z, __uint_as_float(pix));
        bf.st2[nxt][qn] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), s2.z, next_flags);
    } else {
        bf.retire[target & ~kRetireTarget] = make_float4(L.x, L.y, L.z, __uint_as_float(pix));
        if (gv.train) gv.retire_rec[target & ~kRetireTarget] = rec;
        regenerate(rv, bf, nxt);
    }
}

// Any-hit test of the wave's shadow rays (persistent warps, counter cnt[5]); an unoccluded
// ray adds its contribution to the path it belongs to.
__global__ void __launch_bounds__(kB, RTB_TRAV_MIN_BLOCKS) k_shadow(RenderView rv, Buffers bf, int nxt, GuideView gv)
{
    const uint32_t n = min(bf.cnt[2], bf.scap);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(cnt64(bf.cnt, 12), (unsigned long long)n);  // stats
    persistent_traverse(
        rv.sv, n, bf.cnt + 5, true,
        [&](uint32_t i, Trav &T) {
            const float4 r0 = reinterpret_cast<const float4 *>(bf.srays)[2 * i];
            const float4 r1 = reinterpret_cast<const float4 *>(bf.srays)[2 * i + 1];
            const uint32_t sub = __float_as_uint(r1.w) >> kShadowSceneShift;
            trav_init(T, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, r0.w, scene_root(rv.sv, sub));
            T.shadow = (__float_as_uint(r1.w) & 1u) != 0;
        },
        [&](uint32_t i, Trav &T) {
            const float tmax = T.w.tmax;
            bool occ = T.best.prim >= 0 && T.best.t < tmax;
            if (!occ && rv.sv.nspheres) {
                float t = tmax;
                int32_t prim = -1;
                float b1 = 0, b2 = 0;
                const uint32_t sub =
                    __float_as_uint(reinterpret_cast<const float4 *>(bf.srays)[2 * i + 1].w) >> kShadowSceneShift;
                intersect_spheres(rv.sv, sub, T.w.ox, T.w.oy, T.w.oz, T.dx, T.dy, T.dz, tmax, T.shadow, t, prim, b1,
                                  b2);
                occ = prim >= 0 && t < tmax;
            }
            if (occ) return;
            const float4 c = bf.scontrib[i];
            const uint32_t target = __float_as_uint(c.w);
            float *dst = (target & kRetireTarget) ? reinterpret_cast<float *>(bf.retire + (target & ~kRetireTarget))
                                                   : reinterpret_cast<float *>(bf.st1[nxt] + target);
            atomicAdd(dst + 0, c.x);
            atomicAdd(dst + 1, c.y);
            atomicAdd(dst + 2, c.z);
            if (gv.train) {
                const uint32_t rec = (__float_as_uint(reinterpret_cast<const float4 *>(bf.srays)[2 * i + 1].w) >> 1) &
                                     kRecNone;
                if (rec != kRecNone) {
                    float4 *e = &gv.recs[rec].e;
                    atomicAdd(&e->x, c.x);
                    atomicAdd(&e->y, c.y);
                    atomicAdd(&e->z, c.z);
                }
            }
        });
}

// Photon-map gathers queued by k_shade: the density estimate (Scene::combinePhotonContributions,
// zero on subsurface materials, Scene.cu:611-612) or the subsurface dipole estimate
// (Scene::combinePhotonsSubsurface), times the request's weight, added to the path's radiance
// and, while the guide trains, to the guide record of the vertex before it (as k_shadow does).
// One warp per request; warps take requests from counter cnt[7] until the wave's are done.
constexpr int kGatherBlock = 128;
// Resident blocks per SM k_gather is compiled for (64 registers). Config-4 render at 3840x2160,
// 4 spp: 538 / 513 / 464 / 467 ms for no bound (118 registers) / 5 / 6 / 8.
#ifndef RTB_GATHER_MIN_BLOCKS
#define RTB_GATHER_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(kGatherBlock, RTB_GATHER_MIN_BLOCKS) k_gather(RenderView rv, Buffers bf, PhotonView pv, int nxt,
                                                         GuideView gv)
{
    __shared__ PhotonWarpScratch scratch[kGatherBlock / 32];
    PhotonWarpScratch &sm = scratch[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = min(bf.cnt[6], bf.gcap);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(cnt64(bf.cnt, 14), (unsigned long long)n);  // stats
    const bool compat = (rv.flags & RT_RENDER_COMPAT) != 0;
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(bf.cnt + 7, 1u);
        i = __shfl_sync(kFullMask, i, 0);
        if (i >= n) return;  // warp-uniform
        const float4 *g = bf.gather + (uint64_t)kGatherWords * i;
        const float4 a = g[0], b = g[1], c = g[2], d = g[3], k = g[4];
        const rt_material &m = rv.mats[min(__float_as_uint(b.w), rv.nmats - 1)];
        const V3 p = v3(a.x, a.y, a.z), nn = v3(b.x, b.y, b.z), wo = v3(c.x, c.y, c.z), kd = v3(k.x, k.y, k.z);
        const uint32_t kind = __float_as_uint(d.w) & 1u, rec = __float_as_uint(d.w) >> 1;
        V3 e;
        if (kind == kGatherSubsurface) {
            e = warp_photon_subsurface(pv.tree, m, kd, p, nn, wo, __float_as_int(a.w), kSubsurfaceRadius, compat, sm);
        } else if (m.type == RT_MAT_SUBSURFACE) {
            e = v3(0, 0, 0);
        } else {
            Bsdf bs = load_bsdf(m);
            bs.color = kd;  // the textured kd the shading point saw
            e = warp_photon_density(pv.tree, bs, p, nn, wo, __float_as_int(a.w), pv.k, pv.radius, compat, sm);
        }
        if (lane == 0) {
            const V3 contrib = v3(d.x, d.y, d.z) * e;
            const uint32_t target = __float_as_uint(c.w);
            float *dst = (target & kRetireTarget) ? reinterpret_cast<float *>(bf.retire + (target & ~kRetireTarget))
                                                  : reinterpret_cast<float *>(bf.st1[nxt] + target);
            atomicAdd(dst + 0, contrib.x);
            atomicAdd(dst + 1, contrib.y);
            atomicAdd(dst + 2, contrib.z);
            if (gv.train && rec != kRecNone && rec < gv.rec_cap) {
                float4 *r = &gv.recs[rec].e;
                atomicAdd(&r->x, contrib.x);
                atomicAdd(&r->y, contrib.y);
                atomicAdd(&r->z, contrib.z);
            }
        }
    }
}

__device__ __forceinline__ float record_weight(const GuideRecord &r)
{
    float s = 0.f;
    if (r.d.y > 0.f) s += r.e.x / r.d.y;
    if (r.d.z > 0.f) s += r.e.y / r.d.z;
    if (r.d.w > 0.f) s += r.e.z / r.d.w;
    return s * (1.f / 3.f);
}

__device__ __forceinline__ void retire_path(const Buffers &bf, float *sum, uint32_t *count, double *sum64,
                                            const GuideView &gv, uint32_t i)
{
    if (gv.train) {
        // the path is complete: each of its records gets the radiance of everything after it
        uint32_t r = gv.retire_rec[i];
        float ax = 0.f, ay = 0.f, az = 0.f;
        for (int guard = 0; r != kRecNone && r < gv.rec_cap && guard < 256; guard++) {
            GuideRecord &R = gv.recs[r];
            ax += R.e.x;
            ay += R.e.y;
            az += R.e.z;
            R.e.x = ax;
            R.e.y = ay;
            R.e.z = az;
            const float w = record_weight(R);
            if (w > 0.f && isfinite(w)) {
                const uint32_t k = append(gv.rcnt + 1);
                if (k < gv.rec_cap) gv.nz[k] = r;
            }
            r = __float_as_uint(R.e.w);
        }
    }
    float4 v = bf.retire[i];
    if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) return;  // pathTracing.cu:473-486
    uint32_t pix = __float_as_uint(v.w);
    atomicAdd(sum + 3 * pix + 0, v.x);
    atomicAdd(sum + 3 * pix + 1, v.y);
    atomicAdd(sum + 3 * pix + 2, v.z);
    atomicAdd(count + pix, 1u);
    if (sum64) {
        atomicAdd(sum64 + 3 * pix + 0, (double)v.x);
        atomicAdd(sum64 + 3 * pix + 1, (double)v.y);
        atomicAdd(sum64 + 3 * pix + 2, (double)v.z);
    }
}

// The wave's retired paths (usually a small part of the capacity) in a grid-stride loop over
// the resident blocks: a grid of the capacity would spend most of its blocks exiting.
__global__ void __launch_bounds__(kB) k_retire(Buffers bf, float *sum, uint32_t *count, double *sum64, GuideView gv)
{
    const uint32_t n = min(bf.cnt[3], bf.cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        retire_path(bf, sum, count, sum64, gv, i);
}

// Guide network at the wave's hits (queue slots of buffer `cur`); writes the decoded mixture
// per slot, alpha = 0 where the vertex is not guided.
__global__ void __launch_bounds__(kInferWarps * 32, 1) k_guide_infer(RenderView rv, Buffers bf, int cur, const uint4 *img,
                                                                   GuideBox box, GuideParams *params, uint32_t max_depth)
{
    // cnt[16]: set when a tensor-core completion wait ran out (checked after every wave group)
    const uint32_t n = min(bf.cnt[cur], bf.cap);
    const bool compat = (rv.flags & RT_RENDER_COMPAT) != 0;
    auto src = [&](uint32_t q, float *out) -> bool {
        const float4 hv = reinterpret_cast<const float4 *>(bf.hits)[q];
        const rt_hit h{hv.x, __float_as_int(hv.y), hv.z, hv.w};
        if (h.prim < 0 || (bf.st2[cur][q].w & kDepthMask) >= max_depth) return false;
        const float4 r0 = reinterpret_cast<const float4 *>(bf.rays[cur])[2 * q];
        const float4 r1 = reinterpret_cast<const float4 *>(bf.rays[cur])[2 * q + 1];
        const V3 d = v3(r1.x, r1.y, r1.z);
        const Surface sf = surface_at(rv, h, v3(r0.x, r0.y, r0.z), d, compat);
        const Bsdf bs = load_bsdf(rv.mats[min(sf.mat, rv.nmats - 1)]);
        if (!guide_vertex(bs, -dot(d, sf.n))) return false;
        out[0] = sf.p.x;
        out[1] = sf.p.y;
        out[2] = sf.p.z;
        out[3] = sf.n.x;
        out[4] = sf.n.y;
        out[5] = sf.n.z;
        out[6] = -d.x;
        out[7] = -d.y;
        out[8] = -d.z;
        return true;
    };
    auto sink = [&](uint32_t q, bool valid, const float *o) {
        if (!valid) {
            params[q].alpha = 0.f;
            return;
        }
        GuideParams P;
        guide_decode(o, P);
        params[q] = P;
    };
    guide_infer_rows(img, box, n, src, sink, bf.cnt + 16);
}

__global__ void k_texture_lookup(RenderView rv, uint32_t id, const float *uv, uint64_t n, float *rgb)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 c = tex_color(rv, id, uv[2 * i], uv[2 * i + 1]);
    rgb[3 * i] = c.x;
    rgb[3 * i + 1] = c.y;
    rgb[3 * i + 2] = c.z;
}

}  // namespace

}  // namespace rtb

using namespace rtb;

// ------------------------------------------------------------------ C ABI

extern "C" {

int rt_scene_set_materials(rt_scene *s, const rt_material *table, uint32_t n)
{
    if (!s || (!table && n)) return fail(RT_ERR_INVALID, "rt_scene_set_materials: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_set_materials: not available on a merged scene");
    for (uint32_t i = 0; i < n; i++)
        if (table[i].type > RT_MAT_PLASTIC) return fail(RT_ERR_UNSUPPORTED, "rt_scene_set_materials: unknown type");
    s->materials.assign(table, table + n);
    s->render_dirty = true;
    return RT_OK;
}

int rt_scene_set_triangle_materials(rt_scene *s, uint32_t first, uint32_t n, const uint32_t *mats)
{
    if (!s || (!mats && n)) return fail(RT_ERR_INVALID, "rt_scene_set_triangle_materials: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_set_triangle_materials: not available on a merged scene");
    if ((uint64_t)first + n > s->tri_material.size())
        return fail(RT_ERR_INVALID, "rt_scene_set_triangle_materials: range out of bounds");
    std::memcpy(s->tri_material.data() + first, mats, 4ull * n);
    s->render_dirty = true;
    return RT_OK;
}

int rt_render_set_photon_map(rt_scene *s, rt_photon_map *m, uint32_t k, float radius)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_render_set_photon_map: null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_render_set_photon_map: not available on a merged scene");
    if (m && (k == 0 || k > kKnnMaxK)) return fail(RT_ERR_INVALID, "rt_render_set_photon_map: k must be in [1, 128]");
    s->pmap = m;
    s->pm_k = k;
    s->pm_radius = radius;
    return RT_OK;
}

int rt_scene_add_texture(rt_scene *s, const float *rgb, uint32_t width, uint32_t height, uint32_t *id)
{
    if (!s || !rgb || !id) return fail(RT_ERR_INVALID, "rt_scene_add_texture: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_add_texture: not available on a merged scene");
    if (width == 0 || height == 0 || width >= (1u << 24) || height >= (1u << 24) ||
        (uint64_t)width * height >= (1ull << 32))
        return fail(RT_ERR_INVALID, "rt_scene_add_texture: size must be in [1, 2^24) per axis, < 2^32 texels");
    if (s->texels.size() + (uint64_t)width * height >= (1ull << 32))
        return fail(RT_ERR_INVALID, "rt_scene_add_texture: more than 2^32 texels in the scene");
    const uint32_t first = (uint32_t)s->texels.size();
    s->texels.reserve(s->texels.size() + (size_t)width * height);
    for (uint64_t i = 0; i < (uint64_t)width * height; i++)
        s->texels.push_back(make_float4(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], 0.f));
    *id = (uint32_t)s->tex_info.size();
    s->tex_info.push_back(make_uint4(first, width, height, 0u));
    s->tex_dirty = true;
    s->render_dirty = true;
    return RT_OK;
}

int rt_scene_set_triangle_uvs(rt_scene *s, uint32_t first, uint32_t n, const float *uv)
{
    if (!s || (!uv && n)) return fail(RT_ERR_INVALID, "rt_scene_set_triangle_uvs: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_set_triangle_uvs: not available on a merged scene");
    const uint64_t ntri = s->tri9.size() / 9;
    if ((uint64_t)first + n > ntri) return fail(RT_ERR_INVALID, "rt_scene_set_triangle_uvs: range out of bounds");
    if (s->tri_uv.size() < 6 * ntri) {
        const size_t old = s->tri_uv.size() / 6;
        s->tri_uv.resize(6 * ntri);
        for (size_t t = old; t < ntri; t++) {
            float *u = s->tri_uv.data() + 6 * t;
            u[0] = 0.f, u[1] = 0.f, u[2] = 1.f, u[3] = 0.f, u[4] = 1.f, u[5] = 1.f;
        }
    }
    std::memcpy(s->tri_uv.data() + 6ull * first, uv, 24ull * n);
    s->render_dirty = true;
    return RT_OK;
}

int rt_texture_lookup(rt_scene *s, uint32_t id, const float *uv, uint64_t n, float *rgb)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_texture_lookup: null scene");
    if (id >= s->tex_info.size()) return fail(RT_ERR_INVALID, "rt_texture_lookup: unknown texture");
    if (n == 0) return RT_OK;
    if (!uv || !rgb) return fail(RT_ERR_INVALID, "rt_texture_lookup: null buffer");
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    RTB_CHECK(upload_textures(s));
    RenderView rv{};
    rv.texels = s->d_texels.as<float4>();
    rv.tex_info = s->d_tex_info.as<uint4>();
    rv.ntex = (uint32_t)s->tex_info.size();
    const uint64_t blocks = (n + 255) / 256;
    if (blocks >= (1ull << 31)) return fail(RT_ERR_INVALID, "rt_texture_lookup: n too large");
    k_texture_lookup<<<(unsigned)blocks, 256, 0, s->ctx->stream>>>(rv, id, uv, n, rgb);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaStreamSynchronize(s->ctx->stream));
    return RT_OK;
}

int rt_scene_add_point_light(rt_scene *s, const float pos[3], const float rgb[3], float intensity)
{
    if (!s || !pos || !rgb) return fail(RT_ERR_INVALID, "rt_scene_add_point_light: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_add_point_light: not available on a merged scene");
    s->plights.push_back(make_float4(pos[0], pos[1], pos[2], 0.f));
    s->plights.push_back(make_float4(rgb[0] * intensity, rgb[1] * intensity, rgb[2] * intensity, 0.f));
    s->plight_rgbi.push_back({rgb[0], rgb[1], rgb[2], intensity});
    s->render_dirty = true;
    return RT_OK;
}

}  // extern "C"

namespace rtb {

// Uploads what the shading kernels need (materials, per-triangle data, emitters, lights).
void RenderScratch::release()
{
    for (DevBuf *b : {&rays[0], &rays[1], &st0[0], &st0[1], &st1[0], &st1[1], &st2[0], &st2[1], &hits, &srays,
                      &scontrib, &retire, &cnt, &gather, &views, &view_sample0, &view_pixel0, &perm})
        b->release();
    if (host_cnt) cudaFreeHost(host_cnt);
    host_cnt = nullptr;
}

int refresh_transparency(rt_scene *s)
{
    cudaStream_t st = s->ctx->stream;
    auto mat_transparent = [&](uint32_t m) {
        return m < s->materials.size() && (s->materials[m].flags & RT_MATF_TRANSPARENT) != 0;
    };
    RTB_CHECK(refresh_record_flags(s));
    bool schanged = false;
    for (auto &sp : s->spheres) {
        uint32_t f = ((sp.flags & 2u) || mat_transparent(sp.material)) ? 1u : 0u;
        uint32_t nf = (sp.flags & ~1u) | f;
        if (nf != sp.flags) {
            sp.flags = nf;
            schanged = true;
        }
    }
    if (schanged) RTB_CHECK(s->d_spheres.upload(s->spheres.data(), s->spheres.size() * sizeof(SphereRecord), st));
    return RT_OK;
}

// texels and texture table, when textures were added since the last upload
int upload_textures(rt_scene *s)
{
    if (!s->tex_dirty) return RT_OK;
    cudaStream_t st = s->ctx->stream;
    if (!s->texels.empty()) {
        RTB_CHECK(s->d_texels.upload(s->texels.data(), sizeof(float4) * s->texels.size(), st));
        RTB_CHECK(s->d_tex_info.upload(s->tex_info.data(), sizeof(uint4) * s->tex_info.size(), st));
    }
    s->tex_dirty = false;
    return RT_OK;
}

int upload_render_data(rt_scene *s)
{
    if (!s->render_dirty) return RT_OK;
    cudaStream_t st = s->ctx->stream;
    RTB_CHECK(refresh_transparency(s));
    const uint32_t n = (uint32_t)(s->tri9.size() / 9);
    if (s->materials.empty()) return fail(RT_ERR_STATE, "rt_render: no materials set");
    for (uint32_t m : s->tri_material)
        if (m >= s->materials.size()) return fail(RT_ERR_INVALID, "rt_render: triangle material id out of range");
    for (const auto &sp : s->spheres)
        if (sp.material >= s->materials.size()) return fail(RT_ERR_INVALID, "rt_render: sphere material out of range");
    for (const auto &m : s->materials)
        if (m.texture > s->tex_info.size()) return fail(RT_ERR_INVALID, "rt_render: material texture id out of range");
    if (!s->tri_uv.empty() && s->tri_uv.size() < 6ull * n) {  // triangles added after the coordinates
        const size_t old = s->tri_uv.size() / 6;
        s->tri_uv.resize(6ull * n);
        for (size_t t = old; t < n; t++) {
            float *u = s->tri_uv.data() + 6 * t;
            u[0] = 0.f, u[1] = 0.f, u[2] = 1.f, u[3] = 0.f, u[4] = 1.f, u[5] = 1.f;
        }
    }
    if (!s->tri_uv.empty()) RTB_CHECK(s->d_tri_uv.upload(s->tri_uv.data(), 4ull * 6 * n, st));
    RTB_CHECK(upload_textures(s));
    RTB_CHECK(s->d_mats.upload(s->materials.data(), s->materials.size() * sizeof(rt_material), st));
    RTB_CHECK(s->d_tri_mat.upload(s->tri_material.data(), 4ull * n, st));
    bool any_normals = false;
    for (int32_t x : s->tri_normal_idx) any_normals |= x >= 0;
    if (any_normals) {
        RTB_CHECK(s->d_tri_nidx.upload(s->tri_normal_idx.data(), 4ull * s->tri_normal_idx.size(), st));
        RTB_CHECK(s->d_normals.upload(s->normals.data(), 4ull * s->normals.size(), st));
    }
    s->has_normals = any_normals;
    std::vector<uint32_t> etri;
    std::vector<float> cdf;
    double acc = 0;
    uint32_t sub = 0;  // merged scene: emitters are gathered per scene, each cdf from 0
    for (uint32_t t = 0; t < n; t++) {
        if (s->merged) {
            while (sub + 1 < s->sub_tri0.size() && t >= s->sub_tri0[sub + 1]) {
                s->subs[sub].etotal = (float)acc;
                sub++;
                s->subs[sub].e0 = (uint32_t)etri.size();
                acc = 0;
            }
        }
        const rt_material &m = s->materials[s->tri_material[t]];
        if (m.type != RT_MAT_LIGHT) continue;
        const float *p = s->tri9.data() + 9ull * t;
        double ax = p[3] - p[0], ay = p[4] - p[1], az = p[5] - p[2];
        double bx = p[6] - p[0], by = p[7] - p[1], bz = p[8] - p[2];
        double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
        double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        double lum = 0.212671 * m.color[0] * m.intensity + 0.715160 * m.color[1] * m.intensity +
                     0.072169 * m.color[2] * m.intensity;
        if (!(area * lum > 0)) continue;
        acc += area * lum;
        etri.push_back(t);
        cdf.push_back((float)acc);
    }
    s->emit_total = (float)acc;
    s->nemit = (uint32_t)etri.size();
    if (s->merged) {
        for (uint32_t k = sub + 1; k < s->subs.size(); k++) s->subs[k].e0 = (uint32_t)etri.size();  // trailing empty scenes
        s->subs[sub].etotal = (float)acc;
        for (size_t k = 0; k < s->subs.size(); k++) {
            const uint32_t e1 = k + 1 < s->subs.size() ? s->subs[k + 1].e0 : (uint32_t)etri.size();
            s->subs[k].ne = e1 - s->subs[k].e0;
            if (s->subs[k].ne == 0) s->subs[k].etotal = 0.f;
        }
        s->subs[0].e0 = 0;
        RTB_CHECK(s->d_subs.upload(s->subs.data(), s->subs.size() * sizeof(SubScene), st));
    }
    if (!etri.empty()) {
        RTB_CHECK(s->d_emit_tri.upload(etri.data(), 4ull * etri.size(), st));
        RTB_CHECK(s->d_emit_cdf.upload(cdf.data(), 4ull * cdf.size(), st));
    }
    if (!s->plights.empty()) RTB_CHECK(s->d_plights.upload(s->plights.data(), 16ull * s->plights.size(), st));
    RTB_CHECK(s->d_tri_shape.upload(s->tri_shape.data(), 4ull * n, st));
    s->render_dirty = false;
    return RT_OK;
}

int make_render_view(rt_scene *s, RenderView &rv)
{
    RTB_CHECK(upload_render_data(s));
    rv = RenderView{};
    rv.sv = s->view();
    rv.mats = s->d_mats.as<rt_material>();
    rv.nmats = (uint32_t)s->materials.size();
    rv.tri_mat = s->d_tri_mat.as<uint32_t>();
    rv.tri_shape = s->d_tri_shape.as<int32_t>();
    rv.tri_nidx = s->has_normals ? s->d_tri_nidx.as<int32_t>() : nullptr;
    rv.normals = s->has_normals ? s->d_normals.as<float>() : nullptr;
    rv.emit_tri = s->d_emit_tri.as<uint32_t>();
    rv.emit_cdf = s->d_emit_cdf.as<float>();
    rv.nemit = s->nemit;
    rv.emit_total = s->emit_total;
    rv.plights = s->d_plights.as<float4>();
    rv.nplights = (uint32_t)(s->plights.size() / 2);
    rv.texels = s->d_texels.as<float4>();
    rv.tex_info = s->d_tex_info.as<uint4>();
    rv.ntex = (uint32_t)s->tex_info.size();
    rv.tri_uv = s->tri_uv.empty() ? nullptr : s->d_tri_uv.as<float>();
    return RT_OK;
}

}  // namespace rtb

namespace rtb {
namespace {

// Blocks of `kernel` (block size `block`) resident on the current device at once (cached).
template <typename Kernel>
unsigned resident_grid(DeviceSlot slot, Kernel kernel, int block)
{
    unsigned r = device_slot(slot);
    if (!r) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
        r = device_sm_count() * (unsigned)std::max(per_sm, 1);
        set_device_slot(slot, r);
    }
    return r;
}

// Path capacity when the caller gives none: the largest power of two of at most 2^26 paths
// whose wave buffers fit in an eighth of the device's memory; when the call needs more queue
// than the scene holds, also in a quarter of what is free (the queues held count as free, as
// they are reused), so that several scenes in one process shrink each other's default. The
// free-memory query runs only when the queues must grow: it is not free (milliseconds with
// many allocations live). Fewer, larger waves shorten the time the persistent traversal
// kernels spend draining their last rays, wave after wave. BVH-stress render at 1920x1080 x 64
// spp (244 B per path), Mrays/s: 1585 / 1806 / 1947 / 2074 / 2130 / 2189 for 2^21 / 2^22 /
// 2^23 / 2^24 / 2^25 / 2^26 paths.
uint32_t default_paths(uint32_t flags, uint32_t per_path_shadow, uint64_t held_paths, uint64_t samples)
{
    uint64_t bytes = 64 + 96 + 16 + 16 + 4;  // rays, path state, hits, retire, shading order
    bytes += 48ull * std::max<uint32_t>(per_path_shadow, 1);
    if (flags & (RT_RENDER_PHOTON_MAP | RT_RENDER_SUBSURFACE | RT_RENDER_HYBRID)) bytes += 2ull * 16 * kGatherWords;
    if (flags & RT_RENDER_GUIDE) bytes += 208 + 4;
    const uint64_t total_b = (uint64_t)device_mem_mib() << 20;
    uint32_t cap = 1u << 26;
    while (cap > (1u << 20) && (uint64_t)cap * bytes > total_b / 8) cap >>= 1;
    const uint64_t need = std::min<uint64_t>(cap, std::max<uint64_t>(samples, 1024));
    if (need <= held_paths) return cap;  // the queues held already cover the call
    size_t free_b = 0, tb = 0;
    if (cudaMemGetInfo(&free_b, &tb) != cudaSuccess) {
        (void)cudaGetLastError();
        return cap;
    }
    const uint64_t budget = (free_b + held_paths * bytes) / 4;
    while (cap > (1u << 20) && cap > held_paths && std::min<uint64_t>(cap, need) * bytes > budget) cap >>= 1;
    return cap;
}

// Renders the views of one scene in one wavefront (rt_render is a batch of one view).
int render_views(rt_scene *s, const rt_view *views, uint32_t nviews, uint32_t flags, uint32_t max_paths,
                 float *sum_rgb, uint32_t *count, double *sum64, rt_render_stats *stats, const char *who)
{
    const std::string name(who);
    if (!s || !views || nviews == 0 || !sum_rgb || !count) return fail(RT_ERR_INVALID, name + ": null argument");
    if (!s->committed) return fail(RT_ERR_STATE, name + ": scene not committed");
    if (s->merged) {
        if (flags & (RT_RENDER_EXACT_TRACE | RT_RENDER_PHOTON_MAP | RT_RENDER_SUBSURFACE | RT_RENDER_HYBRID))
            return fail(RT_ERR_UNSUPPORTED, name + ": a merged scene renders without photon maps or exact tracing");
        for (uint32_t i = 0; i < nviews; i++)
            if (views[i].scene >= s->subs.size()) return fail(RT_ERR_INVALID, name + ": view scene index out of range");
    } else {
        for (uint32_t i = 0; i < nviews; i++)
            if (views[i].scene != 0) return fail(RT_ERR_INVALID, name + ": view scene index without a merged scene");
    }
    std::vector<uint64_t> sample0(nviews + 1, 0);
    std::vector<uint32_t> pixel0(nviews + 1, 0);
    uint32_t depth_max = 0;
    uint64_t pixels = 0;
    for (uint32_t i = 0; i < nviews; i++) {
        const rt_view &v = views[i];
        if (v.camera.width == 0 || v.camera.height == 0 || v.spp == 0 || v.max_depth == 0)
            return fail(RT_ERR_INVALID, name + ": empty image, spp or depth");
        if (v.max_depth > 255) return fail(RT_ERR_INVALID, name + ": max_depth above 255");
        const uint64_t np = (uint64_t)v.camera.width * v.camera.height;
        pixels += np;
        if (pixels >= (1ull << 31)) return fail(RT_ERR_INVALID, name + ": images too large");
        sample0[i + 1] = sample0[i] + np * v.spp;
        pixel0[i + 1] = (uint32_t)pixels;
        depth_max = std::max(depth_max, v.max_depth);
    }
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    const uint64_t total = sample0[nviews];
    RenderScratch &rs = s->rscratch;
    RTB_CHECK(rs.views.upload(views, sizeof(rt_view) * nviews, st));
    RTB_CHECK(rs.view_sample0.upload(sample0.data(), 8ull * (nviews + 1), st));
    RTB_CHECK(rs.view_pixel0.upload(pixel0.data(), 4ull * (nviews + 1), st));
    const uint32_t per_path_shadow = (uint32_t)(s->plights.size() / 2) + ((flags & RT_RENDER_NEE_AREA) ? 1 : 0);
    uint32_t cap = max_paths ? max_paths : default_paths(flags, per_path_shadow, rs.rays[0].bytes / 32, total);
    cap = (uint32_t)std::min<uint64_t>(cap, std::max<uint64_t>(total, 1024));
    cap = (cap + kB - 1) / kB * kB;
    const uint32_t scap = std::max<uint32_t>(cap * std::max<uint32_t>(per_path_shadow, 1), kB);
    RTB_CHECK(rs.rays[0].reserve(32ull * cap));
    RTB_CHECK(rs.rays[1].reserve(32ull * cap));
    for (int b = 0; b < 2; b++) {
        RTB_CHECK(rs.st0[b].reserve(16ull * cap));
        RTB_CHECK(rs.st1[b].reserve(16ull * cap));
        RTB_CHECK(rs.st2[b].reserve(16ull * cap));
    }
    RTB_CHECK(rs.hits.reserve(16ull * cap));
    RTB_CHECK(rs.srays.reserve(32ull * scap));
    RTB_CHECK(rs.scontrib.reserve(16ull * scap));
    RTB_CHECK(rs.retire.reserve(16ull * cap));
    const bool gathers = (flags & (RT_RENDER_PHOTON_MAP | RT_RENDER_SUBSURFACE | RT_RENDER_HYBRID)) != 0;
    // a path queues at most two gathers per wave (density, subsurface)
    const uint32_t gcap = gathers ? 2 * cap : 0;
    if (gathers) {
        if (!s->pmap || !s->pmap->built)
            return fail(RT_ERR_STATE, name + ": photon-map modes need a built photon map (rt_render_set_photon_map)");
        RTB_CHECK(rs.gather.reserve(16ull * kGatherWords * gcap));
    }
    const bool guided = (flags & RT_RENDER_GUIDE) != 0;
    GuideView gv{};
    rt_guide *guide = s->guide;
    if (guided) {
        if (!guide) return fail(RT_ERR_STATE, name + ": RT_RENDER_GUIDE needs a guide (rt_render_set_guide)");
        // photon-mapping mode ends each path at its first scattering vertex, where the guide
        // would sample: nothing is left to guide
        if (flags & RT_RENDER_PHOTON_MAP)
            return fail(RT_ERR_UNSUPPORTED, name + ": RT_RENDER_GUIDE with RT_RENDER_PHOTON_MAP");
        gv.enabled = 1;
        gv.train = s->guide_train;
        gv.max_depth = guide->opts.max_depth ? guide->opts.max_depth : 0xFFFFFFFFu;
        if (guide->trained) {
            RTB_CHECK(guide->params.reserve(sizeof(GuideParams) * (uint64_t)cap));
            gv.params = guide->params.as<GuideParams>();
        }
        if (gv.train) {
            RTB_CHECK(guide->recs.reserve(sizeof(GuideRecord) * (uint64_t)guide->rec_cap));
            RTB_CHECK(guide->nz.reserve(4ull * guide->rec_cap));
            RTB_CHECK(guide->retire_rec.reserve(4ull * cap));
            RTB_CHECK(guide->rcnt.reserve(16));
            RTB_CUDA(cudaMemsetAsync(guide->rcnt.ptr, 0, 16, st));
            gv.recs = guide->recs.as<GuideRecord>();
            gv.nz = guide->nz.as<uint32_t>();
            gv.retire_rec = guide->retire_rec.as<uint32_t>();
            gv.rcnt = guide->rcnt.as<uint32_t>();
            gv.rec_cap = guide->rec_cap;
        }
    }
    RTB_CHECK(rs.cnt.reserve(256));
    RTB_CHECK(s->scratch.queue.reserve(4ull * cap));
    RTB_CHECK(s->scratch.counters.reserve(64));
    if (!rs.host_cnt) RTB_CUDA(cudaMallocHost(&rs.host_cnt, 256));

    Buffers bf;
    for (int b = 0; b < 2; b++) {
        bf.rays[b] = rs.rays[b].as<rt_ray>();
        bf.st0[b] = rs.st0[b].as<float4>();
        bf.st1[b] = rs.st1[b].as<float4>();
        bf.st2[b] = rs.st2[b].as<uint4>();
    }
    bf.hits = rs.hits.as<rt_hit>();
    bf.srays = rs.srays.as<rt_ray>();
    bf.scontrib = rs.scontrib.as<float4>();
    bf.retire = rs.retire.as<float4>();
    bf.gather = rs.gather.as<float4>();
    PhotonView pv{};
    if (gathers) {
        pv.tree = photon_tree(s->pmap);
        pv.k = std::min<uint32_t>(std::max<uint32_t>(s->pm_k, 1u), kKnnMaxK);
        pv.radius = s->pm_radius;
    }
    bf.cap = cap;
    bf.scap = scap;
    bf.gcap = gcap;
    // material sort of the shading order, chunks of 2^sort_log2 queue slots (0: off)
    const uint32_t sort_log2 = s->sort_log2 ? std::min<uint32_t>(std::max<uint32_t>(s->sort_log2, 5u), kSortMaxLog2) : 0u;
    const unsigned sort_blocks =
        sort_log2 ? std::min((unsigned)((cap + (1u << sort_log2) - 1) >> sort_log2),
                             resident_grid(SLOT_SORT_RESIDENT, k_material_sort, kSortBlock))
                  : 0u;
    if (sort_log2) RTB_CHECK(rs.perm.reserve(4ull * cap));
    bf.perm = sort_log2 ? rs.perm.as<uint32_t>() : nullptr;
    bf.cnt = rs.cnt.as<uint32_t>();

    RenderView rv{};
    RTB_CHECK(make_render_view(s, rv));
    rv.views = rs.views.as<rt_view>();
    rv.view_sample0 = rs.view_sample0.as<uint64_t>();
    rv.view_pixel0 = rs.view_pixel0.as<uint32_t>();
    rv.nviews = nviews;
    rv.flags = flags;
    rv.total = total;

    cudaEvent_t e0, e1;
    RTB_CUDA(cudaEventCreate(&e0));
    RTB_CUDA(cudaEventCreate(&e1));
    RTB_CUDA(cudaEventRecord(e0, st));
    RTB_CUDA(cudaMemsetAsync(bf.cnt, 0, 256, st));
    const unsigned blocks = cap / kB;
    const unsigned retire_blocks = std::min(blocks, resident_grid(SLOT_RETIRE_RESIDENT, k_retire, kB));
    const unsigned shadow_blocks =
        std::min<unsigned>(resident_grid(SLOT_SHADOW_RESIDENT, k_shadow, kB), (scap + kB - 1) / kB);
    unsigned gather_resident = device_slot(SLOT_GATHER_RESIDENT);  // persistent gather warps: every resident block
    if (gathers && !gather_resident) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather, kGatherBlock, 0);
        gather_resident = device_sm_count() * (unsigned)std::max(per_sm, 1);
        set_device_slot(SLOT_GATHER_RESIDENT, gather_resident);
    }
    const unsigned gather_blocks =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(gather_resident, ((uint64_t)gcap * 32 + kGatherBlock - 1) /
                                                                                kGatherBlock));
    if (gv.params && !(device_slot(SLOT_SMEM_ATTRS) & SMEM_RENDER_INFER)) {
        RTB_CUDA(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem));
        or_device_slot(SLOT_SMEM_ATTRS, SMEM_RENDER_INFER);
    }
    const unsigned infer_blocks = (unsigned)std::max(1, s->ctx->sm_count);  // one CTA of 4 tile groups per SM
    const GuideBox gbox = guided ? guide_box(guide) : GuideBox{};
    k_start<<<blocks, kB, 0, st>>>(rv, bf);
    RTB_CUDA(cudaGetLastError());
    const uint32_t trace_flags = (flags & RT_RENDER_EXACT_TRACE) ? 0u : RT_TRACE_FAST;
    uint64_t waves = 0;
    const uint64_t max_waves = (uint64_t)depth_max * (total / std::max<uint32_t>(cap / 4, 1) + 8) + 64;
    // RT_RENDER_STAGE_TIMES: an event at each stage boundary of each wave of a group (host loop,
    // no graphs), the elapsed times summed into rs.stage_ms after every group
    const bool stage_times = (flags & RT_RENDER_STAGE_TIMES) != 0;
    for (int k = 0; k < RT_RENDER_STAGES; k++) rs.stage_ms[k] = 0.0;
    struct StageEvents {  // destroyed on every return path
        cudaEvent_t e[4][RT_RENDER_STAGES + 1] = {};
        ~StageEvents()
        {
            for (auto &row : e)
                for (cudaEvent_t ev : row)
                    if (ev) cudaEventDestroy(ev);
        }
    } sev;
    if (stage_times)
        for (auto &row : sev.e)
            for (cudaEvent_t &ev : row) RTB_CUDA(cudaEventCreate(&ev));
    auto mark = [&](int k, int b) -> int {
        if (stage_times) RTB_CUDA(cudaEventRecord(sev.e[k][b], st));
        return RT_OK;
    };
    // One group = 4 waves (cur 0, 1, 0, 1). The first group is launched directly; the rest
    // replay it as a CUDA graph captured from the second group's launches.
    auto wave_group = [&]() -> int {
        int cur = 0;
        for (int k = 0; k < 4; k++) {
            RTB_CHECK(mark(k, 0));
            RTB_CHECK(launch_trace_closest_dev(rv.sv, bf.rays[cur], bf.cnt + cur, cap, bf.hits, trace_flags,
                                               s->scratch.queue.as<uint32_t>(), s->scratch.counters.as<uint32_t>(),
                                               st));
            RTB_CHECK(mark(k, 1));
            if (gv.params) {
                k_guide_infer<<<infer_blocks, kInferWarps * 32, kInferSmem, st>>>(
                    rv, bf, cur, guide->img.as<uint4>(), gbox, guide->params.as<GuideParams>(), gv.max_depth);
                RTB_CUDA(cudaGetLastError());
            }
            RTB_CHECK(mark(k, 2));
            RTB_CUDA(cudaMemsetAsync(bf.cnt + ((cur ^ 1)), 0, 4, st));
            RTB_CUDA(cudaMemsetAsync(bf.cnt + 2, 0, 24, st));
            if (sort_log2) {
                k_material_sort<<<sort_blocks, kSortBlock, 0, st>>>(rv, bf, cur, rs.perm.as<uint32_t>(), sort_log2);
                RTB_CUDA(cudaGetLastError());
            }
            RTB_CHECK(mark(k, 3));
            k_shade<<<blocks, kB, 0, st>>>(rv, bf, cur, gv);
            RTB_CUDA(cudaGetLastError());
            RTB_CHECK(mark(k, 4));
            k_shadow<<<shadow_blocks, kB, 0, st>>>(rv, bf, cur ^ 1, gv);
            RTB_CUDA(cudaGetLastError());
            RTB_CHECK(mark(k, 5));
            if (gathers) {
                k_gather<<<gather_blocks, kGatherBlock, 0, st>>>(rv, bf, pv, cur ^ 1, gv);
                RTB_CUDA(cudaGetLastError());
            }
            RTB_CHECK(mark(k, 6));
            k_retire<<<retire_blocks, kB, 0, st>>>(bf, sum_rgb, count, sum64, gv);
            RTB_CUDA(cudaGetLastError());
            RTB_CHECK(mark(k, 7));
            cur ^= 1;
        }
        return RT_OK;
    };
    cudaGraphExec_t graph = nullptr;
    auto release_graph = [&]() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    };
    // Device-side wave loop: one CUDA graph whose conditional WHILE node repeats the 4-wave
    // group, ended by k_wave_check on the device, so the host waits once per frame instead of
    // after every group. Where conditional graphs cannot be built (the legacy default stream
    // cannot be captured) the host loop below runs instead.
    bool device_loop = false;
    const uint32_t wave_cap = (uint32_t)std::min<uint64_t>(max_waves, 0x7FFFFFF0u);
    if (st != nullptr && st != cudaStreamLegacy && !(flags & (RT_RENDER_HOST_LOOP | RT_RENDER_STAGE_TIMES))) {
        cudaGraph_t g = nullptr;
        cudaGraphConditionalHandle loop_handle;
        bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
                  cudaGraphConditionalHandleCreate(&loop_handle, g, 1u, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraph_t body = nullptr;
        if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = loop_handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t cn;
            ok = cudaGraphAddNode(&cn, g, nullptr, 0, &cp) == cudaSuccess;
            if (ok) body = cp.conditional.phGraph_out[0];
        }
        if (ok && cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                      cudaSuccess) {
            int rc = wave_group();
            if (rc == RT_OK) {
                k_wave_check<<<1, 32, 0, st>>>(bf.cnt, total, wave_cap, loop_handle);
                rc = cuda_status(cudaGetLastError(), "k_wave_check");
            }
            cudaGraph_t captured = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &captured);
            if (rc != RT_OK) {
                cudaGraphDestroy(g);
                return rc;
            }
            ok = ce == cudaSuccess && cudaGraphInstantiate(&graph, g, 0) == cudaSuccess;
        } else {
            ok = false;
        }
        if (g) cudaGraphDestroy(g);
        if (ok) {
            device_loop = true;
        } else {
            release_graph();
            (void)cudaGetLastError();  // fall back to the host loop
        }
    }
    if (device_loop) {
        cudaError_t ce = cudaGraphLaunch(graph, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(rs.host_cnt, bf.cnt, 128, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        release_graph();
        if (ce != cudaSuccess) return cuda_status(ce, "device wave loop");
        const uint32_t *hc = static_cast<const uint32_t *>(rs.host_cnt);
        waves = hc[18];
        if (hc[16]) return fail(RT_ERR_TIMEOUT, name + ": guide tensor-core completion wait timed out");
        if (hc[19]) return fail(RT_ERR_TIMEOUT, name + ": wave cap exceeded");
    }
    for (uint64_t group = 0; !device_loop; group++) {
        int rc = RT_OK;
        // the legacy default stream cannot be captured: there every group is launched directly
        if (group == 1 && !stage_times && st != nullptr && st != cudaStreamLegacy &&
            cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            rc = wave_group();
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (rc == RT_OK && ce == cudaSuccess && g) {
                const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) return cuda_status(ie, "cudaGraphInstantiate");
            } else {
                if (g) cudaGraphDestroy(g);
                if (rc != RT_OK) return rc;
                return cuda_status(ce, "cudaStreamEndCapture");
            }
        }
        if (graph) {
            const cudaError_t le = cudaGraphLaunch(graph, st);
            if (le != cudaSuccess) {
                release_graph();
                return cuda_status(le, "cudaGraphLaunch");
            }
        } else {
            rc = wave_group();
            if (rc != RT_OK) return rc;
        }
        waves += 4;
        cudaError_t ce = cudaMemcpyAsync(rs.host_cnt, bf.cnt, 128, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) {
            release_graph();
            return cuda_status(ce, "wave group");
        }
        if (stage_times) {
            // stage 1 (guide inference) spans boundaries 1-2, stage 2 (sort and counter resets) 2-3, ...
            for (int k = 0; k < 4; k++)
                for (int b = 0; b < RT_RENDER_STAGES; b++) {
                    float t = 0.f;
                    if (cudaEventElapsedTime(&t, sev.e[k][b], sev.e[k][b + 1]) == cudaSuccess) rs.stage_ms[b] += t;
                }
            (void)cudaGetLastError();
        }
        const uint32_t *hc = static_cast<const uint32_t *>(rs.host_cnt);
        uint64_t next_sample;
        std::memcpy(&next_sample, hc + 8, 8);
        if (hc[16]) {
            release_graph();
            return fail(RT_ERR_TIMEOUT, name + ": guide tensor-core completion wait timed out");
        }
        if (hc[0] == 0 && next_sample >= total) break;
        if (waves > max_waves) {
            release_graph();
            return fail(RT_ERR_TIMEOUT, name + ": wave cap exceeded");
        }
    }
    release_graph();
    RTB_CUDA(cudaEventRecord(e1, st));
    RTB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        const uint32_t *hc = static_cast<const uint32_t *>(rs.host_cnt);
        uint64_t v;
        std::memcpy(&v, hc + 10, 8);
        stats->extension_rays = v;
        std::memcpy(&v, hc + 12, 8);
        stats->shadow_rays = v;
        std::memcpy(&v, hc + 8, 8);
        stats->camera_rays = std::min<uint64_t>(v, total);
        std::memcpy(&v, hc + 14, 8);
        stats->gathers = v;
        stats->waves = waves;
        stats->ms = ms;
    }
    return RT_OK;
}

}  // namespace
}  // namespace rtb

extern "C" int rt_render(rt_scene *s, const rt_camera *cam, const rt_render_opts *opts, float *sum_rgb,
                         uint32_t *count, double *sum64, rt_render_stats *stats)
{
    if (!s || !cam || !opts) return fail(RT_ERR_INVALID, "rt_render: null argument");
    rt_view v{};
    v.camera = *cam;
    v.spp = opts->spp;
    v.sample_offset = opts->sample_offset;
    v.max_depth = opts->max_depth;
    v.rr_depth = opts->rr_depth;
    v.seed = opts->seed;
    return render_views(s, &v, 1, opts->flags, opts->max_paths, sum_rgb, count, sum64, stats, "rt_render");
}

extern "C" int rt_render_batch(rt_scene *s, const rt_view *views, uint32_t nviews, uint32_t flags, uint32_t max_paths,
                               float *sum_rgb, uint32_t *count, double *sum64, rt_render_stats *stats)
{
    return render_views(s, views, nviews, flags, max_paths, sum_rgb, count, sum64, stats, "rt_render_batch");
}

extern "C" int rt_render_stage_times(rt_scene *s, double *ms_out, uint32_t n)
{
    if (!s || (!ms_out && n)) return fail(RT_ERR_INVALID, "rt_render_stage_times: null argument");
    if (n > RT_RENDER_STAGES) return fail(RT_ERR_INVALID, "rt_render_stage_times: at most RT_RENDER_STAGES values");
    for (uint32_t k = 0; k < n; k++) ms_out[k] = s->rscratch.stage_ms[k];
    return RT_OK;
}

extern "C" int rt_render_set_sort(rt_scene *s, uint32_t chunk_log2)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_render_set_sort: null scene");
    if (chunk_log2 != 0 && (chunk_log2 < 5 || chunk_log2 > kSortMaxLog2))
        return fail(RT_ERR_INVALID, "rt_render_set_sort: chunk_log2 must be 0 (off) or 5..13");
    s->sort_log2 = chunk_log2;
    return RT_OK;
}
