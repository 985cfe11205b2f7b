// Photon tracing, the photon-map kd-tree and k-nearest-neighbour gathering (sm_100a).
//
// Tracing (integration/photonDispersion.cu:26-192, Scene.cu:989-1026): photons start at
// the point lights and bounce as paths do in the renderer (same surfaces, BSDFs and Russian
// roulette, surface.cuh); at every hit on a scattering material a photon is stored. Paths
// run as waves (all photons of one bounce per wave, closest hits by the BVH8 kernel);
// stored photons are appended with a (path, depth) key and sorted by it at the end, so the
// photon order does not depend on scheduling.
//
// The kd-tree is the reference's implicit balanced tree (kdtree.h:78-108): the element at
// the middle of a range is the node, split on the axis of largest extent, built on the host
// with the same partial ordering. Queries run one thread per query point on the GPU with a
// bounded max-heap of the k best candidates in local memory.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "photon_query.cuh"

namespace rtb {
namespace {

constexpr int kPB = 128;

struct PhotonBuffers {
    rt_ray *rays[2];
    float4 *beta[2];   // path throughput
    float4 *carry[2];  // carried light rgb, path index bits
    uint4 *rng[2];     // rng state lo/hi, -, depth
    rt_hit *hits;
    rt_photon *store;          // unsorted stored photons
    unsigned long long *keys;  // (path << 8) | depth
    uint32_t store_cap;
    uint32_t cap;
    // [0],[1] queue sizes, [2] stored count, [3] status
    uint32_t *cnt;
};

__device__ __forceinline__ Pcg photon_rng(uint64_t path, uint32_t seed)
{
    return pcg_init((uint32_t)path, 0xFFFFFFFFu, seed ^ 0x9E3779B9u);
}

// Light choice proportional to power, as Scene::selectOneRandomLight (Scene.cu:421-438).
__global__ void k_select(RenderView rv, uint64_t n, uint32_t seed, const float *cdf_power, float total,
                         uint32_t *sel, unsigned long long *per_light)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Pcg r = photon_rng(i, seed);
    float u = pcg_float(r);
    uint32_t l = rv.nplights - 1;
    for (uint32_t k = 0; k < rv.nplights; k++) {
        u -= cdf_power[k] / total;
        if (u <= 0) {
            l = k;
            break;
        }
    }
    sel[i] = l;
    // one add per distinct light of the warp: every thread adding to one of a few counters
    // serialised the kernel (1.9 ms for 10M photons and two lights)
    const unsigned peers = __match_any_sync(__activemask(), l);
    if ((int)(threadIdx.x & 31u) == __ffs(peers) - 1) atomicAdd(per_light + l, (unsigned long long)__popc(peers));
}

// PointLight::sampleLight(sampler, n) (PointLight.cu:68-95) and the selection-pdf division
// (Scene.cu:1008-1012): power = I * 4 pi / n_l / p_l, direction uniform on the sphere.
__global__ void k_emit(RenderView rv, uint64_t n, uint32_t seed, const float *power, float total,
                       const uint32_t *sel, const unsigned long long *per_light, PhotonBuffers pb)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Pcg r = photon_rng(i, seed);
    (void)pcg_float(r);  // the selection sample
    const uint32_t l = sel[i];
    float u1 = pcg_float(r), u2 = pcg_float(r);
    float phi = 2 * kPi * u1;
    float th = acosf(2 * u2 - 1);
    float st, ct, sp, cp;
    sincosf(th, &st, &ct);
    sincosf(phi, &sp, &cp);
    V3 d = v3(st * cp, st * sp, ct);
    float4 lp = rv.plights[2 * l], li = rv.plights[2 * l + 1];
    const float pl = power[l] / total;
    const float scale = (4 * kPi) / (float)per_light[l] / pl;
    const uint32_t q = (uint32_t)i;
    reinterpret_cast<float4 *>(pb.rays[0])[2 * q] = make_float4(lp.x, lp.y, lp.z, INFINITY);
    reinterpret_cast<float4 *>(pb.rays[0])[2 * q + 1] = make_float4(d.x, d.y, d.z, 0.f);
    pb.beta[0][q] = make_float4(1.f, 1.f, 1.f, 0.f);
    pb.carry[0][q] = make_float4(li.x * scale, li.y * scale, li.z * scale, __uint_as_float((uint32_t)i));
    pb.rng[0][q] = make_uint4((uint32_t)r.state, (uint32_t)(r.state >> 32), 0u, 0u);
}

__global__ void __launch_bounds__(kPB) k_photon_shade(RenderView rv, PhotonBuffers pb, int cur, uint32_t max_depth,
                                                      uint32_t rr_depth, uint32_t seed, uint32_t flags)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = min(pb.cnt[cur], pb.cap);
    if (q >= n) return;
    const int nxt = cur ^ 1;
    const bool compat = (flags & RT_RENDER_COMPAT) != 0;
    float4 hv = reinterpret_cast<const float4 *>(pb.hits)[q];
    rt_hit h{hv.x, __float_as_int(hv.y), hv.z, hv.w};
    if (h.prim < 0) return;  // escaped
    float4 r0 = reinterpret_cast<const float4 *>(pb.rays[cur])[2 * q];
    float4 r1 = reinterpret_cast<const float4 *>(pb.rays[cur])[2 * q + 1];
    float4 b4 = pb.beta[cur][q], c4 = pb.carry[cur][q];
    uint4 s4 = pb.rng[cur][q];
    V3 o = v3(r0.x, r0.y, r0.z), d = v3(r1.x, r1.y, r1.z);
    V3 beta = v3(b4.x, b4.y, b4.z), carry = v3(c4.x, c4.y, c4.z);
    const uint32_t path = __float_as_uint(c4.w);
    const uint32_t depth = s4.w;
    Pcg rng;
    rng.state = ((uint64_t)s4.y << 32) | s4.x;
    rng.inc = ((((uint64_t)0xFFFFFFFFu << 32) | (seed ^ 0x9E3779B9u)) << 1u) | 1u;
    Surface sf = surface_at(rv, h, o, d, compat);
    const rt_material &m = rv.mats[min(sf.mat, rv.nmats - 1)];
    Bsdf bs = load_bsdf(m);
    const bool scattering = is_scattering(bs);  // from the material's own kd
    if (m.texture) {
        const float2 uv = surface_uv(rv, h, sf);
        texture_bsdf(bs, tex_color(rv, m.texture - 1u, uv.x, uv.y));
    }
    if (scattering) {  // samplePhotonIntersections (photonDispersion.cu:40-54)
        uint32_t slot = append(pb.cnt + 2);
        if (slot < pb.store_cap) {
            V3 pw = carry * beta;
            rt_photon ph;
            ph.pos[0] = sf.p.x;
            ph.pos[1] = sf.p.y;
            ph.pos[2] = sf.p.z;
            ph.shape_id = sf.shape;
            ph.dir[0] = d.x;
            ph.dir[1] = d.y;
            ph.dir[2] = d.z;
            ph.path = path;
            ph.power[0] = pw.x;
            ph.power[1] = pw.y;
            ph.power[2] = pw.z;
            ph.depth = depth;
            ph.normal[0] = sf.n.x;
            ph.normal[1] = sf.n.y;
            ph.normal[2] = sf.n.z;
            ph.reserved = 0.f;
            pb.store[slot] = ph;
            pb.keys[slot] = ((unsigned long long)path << 8) | depth;
        }
    }
    V3 t, bv;
    onb(sf.n, t, bv);
    V3 wow = -d;
    V3 wo = v3(dot(wow, t), dot(wow, bv), dot(wow, sf.n));
    V3 Le = (bs.type == RT_MAT_LIGHT) ? bs.color * m.intensity : v3(0, 0, 0);
    V3 wi;
    float pdf;
    bool delta;
    V3 f = bsdf_sample(bs, wo, rng, compat, wi, pdf, delta);
    carry = carry + beta * Le;  // photonDispersion.cu:64-65
    beta = beta * f;
    bool finished = is_black(f);
    if (!finished && scattering && depth > rr_depth) {  // finishStep (pathTracing.cu:91-102)
        float qrr = fmaxf(0.05f, 1.f - luminance(beta));
        if (pcg_float(rng) < qrr)
            finished = true;
        else
            beta = beta * (1.f / (1.f - qrr));
    }
    if (finished || depth + 1 >= max_depth) return;
    V3 wiw = t * wi.x + bv * wi.y + sf.n * wi.z;
    V3 no = spawn_origin(sf.p, sf.n, sf.perr, wiw);
    uint32_t qn = append(pb.cnt + nxt);
    reinterpret_cast<float4 *>(pb.rays[nxt])[2 * qn] = make_float4(no.x, no.y, no.z, INFINITY);
    reinterpret_cast<float4 *>(pb.rays[nxt])[2 * qn + 1] = make_float4(wiw.x, wiw.y, wiw.z, 0.f);
    pb.beta[nxt][qn] = make_float4(beta.x, beta.y, beta.z, 0.f);
    pb.carry[nxt][qn] = make_float4(carry.x, carry.y, carry.z, __uint_as_float(path));
    pb.rng[nxt][qn] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), 0u, depth + 1);
}

__global__ void k_gather_photons(const rt_photon *src, const uint32_t *order, uint64_t n, rt_photon *dst)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[order[i]];
}

__global__ void k_iota(uint32_t *v, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

// ------------------------------------------------------------------- kNN

__global__ void __launch_bounds__(128) k_knn(const float4 *__restrict__ node_pos, const int2 *__restrict__ node_aux,
                                             uint32_t n, const float *__restrict__ queries,
                                             const int32_t *__restrict__ qshape, uint64_t nq, uint32_t k,
                                             float radius, int32_t *__restrict__ out_idx,
                                             float *__restrict__ out_dist, uint32_t *__restrict__ out_count)
{
    const uint64_t qi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    float hd[kKnnMaxK];
    int32_t hi[kKnnMaxK];
    const uint32_t cnt = knn_query(node_pos, node_aux, n, queries[3 * qi], queries[3 * qi + 1], queries[3 * qi + 2],
                                   qshape ? qshape[qi] : -1, k, radius, hd, hi);
    heap_to_sorted(hd, hi, cnt);
    for (uint32_t j = 0; j < k; j++) {
        out_idx[qi * k + j] = j < cnt ? hi[j] : -1;
        if (out_dist) out_dist[qi * k + j] = j < cnt ? hd[j] : INFINITY;
    }
    out_count[qi] = cnt;
}

// One warp per query (the render's gather kernel uses the same warp functions).
constexpr int kQueryBlock = 128;
// Resident blocks per SM of the query kernels (64 registers): k_density 54 / 64 / 79 M queries/s
// and k_subsurface 4.5 / 4.5 / 5.1 M/s for no bound (80 registers) / 6 / 8, on a 2.1M-photon map.
#ifndef RTB_QUERY_MIN_BLOCKS
#define RTB_QUERY_MIN_BLOCKS 8
#endif

// The photons' shading attributes in tree-slot order, so that a query reads them with the
// positions it scans: power and cos(normal, -direction) (the photon's factor of
// diffusionTermBSSRDF, geometricMath.cu:503-522), and the arrival direction.
__global__ void k_tree_attrs(const int2 *__restrict__ node_aux, const rt_photon *__restrict__ photons, uint64_t n,
                             float4 *__restrict__ pw, float4 *__restrict__ dir)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const rt_photon ph = photons[node_aux[i].y];
    const V3 pn = v3(ph.normal[0], ph.normal[1], ph.normal[2]);
    const V3 wi = -v3(ph.dir[0], ph.dir[1], ph.dir[2]);
    const float cos_i = dot(pn, wi) / (length(pn) * length(wi));
    pw[i] = make_float4(ph.power[0], ph.power[1], ph.power[2], cos_i);
    dir[i] = make_float4(ph.dir[0], ph.dir[1], ph.dir[2], 0.f);
}


// Scene::combinePhotonContributions (Scene.cu:607-635) per query: the k nearest photons on
// the same shape within radius, sum of power * lightScattered(-photon direction), divided by
// pi * (largest neighbour distance)^2.
__global__ void __launch_bounds__(kQueryBlock, RTB_QUERY_MIN_BLOCKS) k_density(PhotonTree tree, rt_material mat, const float *__restrict__ pts,
                                                         const float *__restrict__ nrm, const float *__restrict__ wo,
                                                         const int32_t *__restrict__ shape, uint64_t nq, uint32_t k,
                                                         float radius, float *__restrict__ out)
{
    __shared__ PhotonWarpScratch scratch[kQueryBlock / 32];
    const uint64_t qi = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (qi >= nq) return;  // warp-uniform
    V3 p = v3(pts[3 * qi], pts[3 * qi + 1], pts[3 * qi + 2]);
    V3 nn = normalize(v3(nrm[3 * qi], nrm[3 * qi + 1], nrm[3 * qi + 2]));
    V3 w = v3(wo[3 * qi], wo[3 * qi + 1], wo[3 * qi + 2]);
    V3 c = warp_photon_density(tree, load_bsdf(mat), p, nn, w, shape ? shape[qi] : -1, k, radius, true,
                               scratch[threadIdx.x >> 5]);
    if ((threadIdx.x & 31u) == 0) {
        out[3 * qi] = c.x;
        out[3 * qi + 1] = c.y;
        out[3 * qi + 2] = c.z;
    }
}

__global__ void __launch_bounds__(kQueryBlock, RTB_QUERY_MIN_BLOCKS) k_subsurface(PhotonTree tree, rt_material mat,
                                                            const float *__restrict__ pts,
                                                            const float *__restrict__ nrm,
                                                            const float *__restrict__ wo,
                                                            const int32_t *__restrict__ shape, uint64_t nq,
                                                            float radius, int compat, float *__restrict__ out)
{
    __shared__ PhotonWarpScratch scratch[kQueryBlock / 32];
    const uint64_t qi = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (qi >= nq) return;  // warp-uniform
    const V3 p = v3(pts[3 * qi], pts[3 * qi + 1], pts[3 * qi + 2]);
    const V3 nn = v3(nrm[3 * qi], nrm[3 * qi + 1], nrm[3 * qi + 2]);
    const V3 w = v3(wo[3 * qi], wo[3 * qi + 1], wo[3 * qi + 2]);
    const V3 c = warp_photon_subsurface(tree, mat, v3(mat.color[0], mat.color[1], mat.color[2]), p, nn, w,
                                        shape ? shape[qi] : -1, radius, compat != 0, scratch[threadIdx.x >> 5]);
    if ((threadIdx.x & 31u) == 0) {
        out[3 * qi] = c.x;
        out[3 * qi + 1] = c.y;
        out[3 * qi + 2] = c.z;
    }
}

// ---------------------------------------------------- host kd-tree build

struct KdElem {
    float p[3];
    int32_t shape;
    uint32_t idx;
};

// build_tree (kdtree.h:78-103): bounding box of the range, axis of largest extent (first
// axis on ties), std::nth_element at the middle, recurse on both halves.
void kd_build(std::vector<KdElem> &e, std::vector<uint8_t> &axis, size_t left, size_t right, int depth)
{
    if (right - left <= 1) return;
    float lo[3], hi[3];
    for (int c = 0; c < 3; c++) lo[c] = hi[c] = e[left].p[c];
    for (size_t i = left + 1; i < right; i++)
        for (int c = 0; c < 3; c++) {
            if (lo[c] > e[i].p[c]) lo[c] = e[i].p[c];
            if (hi[c] < e[i].p[c]) hi[c] = e[i].p[c];
        }
    const size_t median = (right + left) / 2;
    int ax = 0;
    float mx = hi[0] - lo[0];
    for (int c = 1; c < 3; c++)
        if (hi[c] - lo[c] > mx) {
            ax = c;
            mx = hi[c] - lo[c];
        }
    std::nth_element(e.begin() + left, e.begin() + median, e.begin() + right,
                     [ax](const KdElem &a, const KdElem &b) { return a.p[ax] < b.p[ax]; });
    axis[median] = (uint8_t)ax;
    if (right - left > 400000 && depth < 4) {
        std::thread t([&, left, median, depth]() { kd_build(e, axis, left, median, depth + 1); });
        kd_build(e, axis, median + 1, right, depth + 1);
        t.join();
    } else {
        kd_build(e, axis, left, median, depth + 1);
        kd_build(e, axis, median + 1, right, depth + 1);
    }
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

int rt_photon_map_destroy(rt_photon_map *m)
{
    if (!m) return RT_OK;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    m->photons.release();
    m->node_pos.release();
    m->node_aux.release();
    m->node_pw.release();
    m->node_dir.release();
    delete m;
    return RT_OK;
}

int rt_photon_map_count(rt_photon_map *m, uint64_t *n)
{
    if (!m || !n) return fail(RT_ERR_INVALID, "rt_photon_map_count: null argument");
    *n = m->n;
    return RT_OK;
}

int rt_photon_map_get(rt_photon_map *m, uint64_t first, uint64_t n, rt_photon *out)
{
    if (!m || (!out && n)) return fail(RT_ERR_INVALID, "rt_photon_map_get: null argument");
    if (first + n > m->n) return fail(RT_ERR_INVALID, "rt_photon_map_get: range out of bounds");
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaSetDevice(m->ctx->device));
    RTB_CUDA(cudaMemcpyAsync(out, m->photons.as<rt_photon>() + first, n * sizeof(rt_photon), cudaMemcpyDeviceToHost,
                             m->ctx->stream));
    RTB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return RT_OK;
}

int rt_photon_map_from_points(rt_context *ctx, const float *pos, const int32_t *shape, uint64_t n,
                              rt_photon_map **out)
{
    if (!ctx || !out || (!pos && n)) return fail(RT_ERR_INVALID, "rt_photon_map_from_points: null argument");
    if (n >= 0xFFFFFFFFull) return fail(RT_ERR_INVALID, "rt_photon_map_from_points: too many points");
    RTB_CUDA(cudaSetDevice(ctx->device));
    std::vector<float> hp(3 * n);
    std::vector<int32_t> hs(n, -1);
    if (n) {
        RTB_CUDA(cudaMemcpyAsync(hp.data(), pos, 12 * n, cudaMemcpyDeviceToHost, ctx->stream));
        if (shape) RTB_CUDA(cudaMemcpyAsync(hs.data(), shape, 4 * n, cudaMemcpyDeviceToHost, ctx->stream));
        RTB_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    std::vector<rt_photon> ph(n);
    for (uint64_t i = 0; i < n; i++) {
        std::memset(&ph[i], 0, sizeof(rt_photon));
        ph[i].pos[0] = hp[3 * i];
        ph[i].pos[1] = hp[3 * i + 1];
        ph[i].pos[2] = hp[3 * i + 2];
        ph[i].shape_id = hs[i];
        ph[i].path = (uint32_t)i;
    }
    rt_photon_map *m = new rt_photon_map();
    m->ctx = ctx;
    m->n = n;
    int st = m->photons.upload(ph.data(), n * sizeof(rt_photon), ctx->stream);
    if (st != RT_OK) {
        delete m;
        return st;
    }
    *out = m;
    return RT_OK;
}

int rt_photon_map_build(rt_photon_map *m)
{
    if (!m) return fail(RT_ERR_INVALID, "rt_photon_map_build: null map");
    RTB_CUDA(cudaSetDevice(m->ctx->device));
    cudaStream_t st = m->ctx->stream;
    const uint64_t n = m->n;
    std::vector<rt_photon> ph(n);
    if (n) {
        RTB_CUDA(cudaMemcpyAsync(ph.data(), m->photons.ptr, n * sizeof(rt_photon), cudaMemcpyDeviceToHost, st));
        RTB_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<KdElem> e(n);
    for (uint64_t i = 0; i < n; i++) {
        e[i].p[0] = ph[i].pos[0];
        e[i].p[1] = ph[i].pos[1];
        e[i].p[2] = ph[i].pos[2];
        e[i].shape = ph[i].shape_id;
        e[i].idx = (uint32_t)i;
    }
    std::vector<uint8_t> axis(n, 0);
    kd_build(e, axis, 0, n, 0);
    std::vector<float4> np(n);
    std::vector<int2> na(n);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t ax = axis[i];
        float axf;
        std::memcpy(&axf, &ax, 4);
        np[i] = make_float4(e[i].p[0], e[i].p[1], e[i].p[2], axf);
        na[i] = make_int2(e[i].shape, (int)e[i].idx);
    }
    RTB_CHECK(m->node_pos.upload(np.data(), n * sizeof(float4), st));
    RTB_CHECK(m->node_aux.upload(na.data(), n * sizeof(int2), st));
    RTB_CHECK(m->node_pw.reserve(std::max<uint64_t>(n, 1) * sizeof(float4)));
    RTB_CHECK(m->node_dir.reserve(std::max<uint64_t>(n, 1) * sizeof(float4)));
    if (n) {
        k_tree_attrs<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(m->node_aux.as<int2>(), m->photons.as<rt_photon>(), n,
                                                                 m->node_pw.as<float4>(), m->node_dir.as<float4>());
        RTB_CUDA(cudaGetLastError());
    }
    RTB_CUDA(cudaStreamSynchronize(st));
    m->built = true;
    return RT_OK;
}

int rt_photon_knn(rt_photon_map *m, const float *q, const int32_t *qs, uint64_t nq, uint32_t k, float radius,
                  int32_t *out_idx, float *out_dist, uint32_t *out_count)
{
    if (!m || (nq && (!q || !out_idx || !out_count))) return fail(RT_ERR_INVALID, "rt_photon_knn: null argument");
    if (!m->built) return fail(RT_ERR_STATE, "rt_photon_knn: map not built (rt_photon_map_build)");
    if (k == 0 || k > kKnnMaxK) return fail(RT_ERR_INVALID, "rt_photon_knn: k must be in [1, 128]");
    if (nq == 0) return RT_OK;
    RTB_CUDA(cudaSetDevice(m->ctx->device));
    const uint64_t blocks = (nq + 127) / 128;
    k_knn<<<(unsigned)blocks, 128, 0, m->ctx->stream>>>(m->node_pos.as<float4>(), m->node_aux.as<int2>(),
                                                        (uint32_t)m->n, q, qs, nq, k, radius, out_idx, out_dist,
                                                        out_count);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return RT_OK;
}

int rt_photon_subsurface(rt_photon_map *m, const rt_material *mat, const float *pts, const float *nrm, const float *wo,
                         const int32_t *shape, uint64_t nq, float radius, uint32_t flags, float *out_rgb)
{
    if (!m || !mat) return fail(RT_ERR_INVALID, "rt_photon_subsurface: null argument");
    if (!m->built) return fail(RT_ERR_STATE, "rt_photon_subsurface: photon map not built");
    if (mat->type != RT_MAT_SUBSURFACE) return fail(RT_ERR_INVALID, "rt_photon_subsurface: not a subsurface material");
    if (nq == 0) return RT_OK;
    if (!pts || !nrm || !wo || !out_rgb) return fail(RT_ERR_INVALID, "rt_photon_subsurface: null buffer");
    RTB_CUDA(cudaSetDevice(m->ctx->device));
    if (nq > (1ull << 31) / 32) return fail(RT_ERR_INVALID, "rt_photon_subsurface: nq must be at most 2^26");
    const uint64_t blocks = (nq * 32 + kQueryBlock - 1) / kQueryBlock;
    k_subsurface<<<(unsigned)blocks, kQueryBlock, 0, m->ctx->stream>>>(photon_tree(m), *mat, pts, nrm, wo, shape, nq,
                                                                       radius, (flags & RT_RENDER_COMPAT) ? 1 : 0,
                                                                       out_rgb);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return RT_OK;
}

int rt_photon_density(rt_photon_map *m, const rt_material *mat, const float *pts, const float *nrm, const float *wo,
                      const int32_t *shape, uint64_t nq, uint32_t k, float radius, float *out_rgb)
{
    if (!m || !mat || (nq && (!pts || !nrm || !wo || !out_rgb)))
        return fail(RT_ERR_INVALID, "rt_photon_density: null argument");
    if (!m->built) return fail(RT_ERR_STATE, "rt_photon_density: map not built (rt_photon_map_build)");
    if (k == 0 || k > kKnnMaxK) return fail(RT_ERR_INVALID, "rt_photon_density: k must be in [1, 128]");
    if (nq == 0) return RT_OK;
    RTB_CUDA(cudaSetDevice(m->ctx->device));
    if (nq > (1ull << 31) / 32) return fail(RT_ERR_INVALID, "rt_photon_density: nq must be at most 2^26");
    const uint64_t blocks = (nq * 32 + kQueryBlock - 1) / kQueryBlock;
    k_density<<<(unsigned)blocks, kQueryBlock, 0, m->ctx->stream>>>(photon_tree(m), *mat, pts, nrm, wo, shape, nq, k,
                                                                    radius, out_rgb);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return RT_OK;
}

int rt_photons_trace(rt_scene *s, uint64_t n, uint32_t max_depth, uint32_t rr_depth, uint32_t seed, uint32_t flags,
                     rt_photon_map **out, rt_photon_trace_stats *stats)
{
    if (!s || !out) return fail(RT_ERR_INVALID, "rt_photons_trace: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_photons_trace: not available on a merged scene");
    if (!s->committed) return fail(RT_ERR_STATE, "rt_photons_trace: scene not committed");
    if (n == 0 || n >= (1ull << 31)) return fail(RT_ERR_INVALID, "rt_photons_trace: n must be in [1, 2^31)");
    if (max_depth == 0 || max_depth > 255) return fail(RT_ERR_INVALID, "rt_photons_trace: max_depth in [1, 255]");
    if (s->plights.empty()) return fail(RT_ERR_STATE, "rt_photons_trace: the scene has no point lights");
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    RenderView rv;
    RTB_CHECK(make_render_view(s, rv));
    const uint32_t nl = (uint32_t)s->plight_rgbi.size();
    std::vector<float> power(nl);
    float total = 0.f;
    for (uint32_t l = 0; l < nl; l++) {  // sum(Light::power()) = sum(color * I * 4 pi) (PointLight.cu:40-43)
        const auto &p = s->plight_rgbi[l];
        power[l] = (p.r * p.i * 4.0f * kPi) + (p.g * p.i * 4.0f * kPi) + (p.b * p.i * 4.0f * kPi);
        total += power[l];
    }
    if (!(total > 0)) return fail(RT_ERR_STATE, "rt_photons_trace: lights have no power");
    const uint32_t cap = (uint32_t)n;
    DevBuf rays[2], beta[2], carry[2], rng[2], hits, sel, perl, dpow, cnt, queue;  // freed on return
    for (int b = 0; b < 2; b++) {
        RTB_CHECK(rays[b].reserve(32ull * cap));
        RTB_CHECK(beta[b].reserve(16ull * cap));
        RTB_CHECK(carry[b].reserve(16ull * cap));
        RTB_CHECK(rng[b].reserve(16ull * cap));
    }
    RTB_CHECK(hits.reserve(16ull * cap));
    RTB_CHECK(sel.reserve(4ull * cap));
    RTB_CHECK(perl.reserve(8ull * nl));
    RTB_CHECK(dpow.upload(power.data(), 4ull * nl, st));
    RTB_CHECK(cnt.reserve(64));
    RTB_CHECK(queue.reserve(4ull * cap));
    RTB_CHECK(s->scratch.counters.reserve(64));
    uint64_t store_cap = std::max<uint64_t>(4 * n, 1024);
    rt_photon_map *m = nullptr;
    cudaEvent_t e0, e1;
    RTB_CUDA(cudaEventCreate(&e0));
    RTB_CUDA(cudaEventCreate(&e1));
    uint64_t stored = 0, rays_traced = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        DevBuf store, keys;
        RTB_CHECK(store.reserve(sizeof(rt_photon) * store_cap));
        RTB_CHECK(keys.reserve(8 * store_cap));
        PhotonBuffers pb;
        for (int b = 0; b < 2; b++) {
            pb.rays[b] = rays[b].as<rt_ray>();
            pb.beta[b] = beta[b].as<float4>();
            pb.carry[b] = carry[b].as<float4>();
            pb.rng[b] = rng[b].as<uint4>();
        }
        pb.hits = hits.as<rt_hit>();
        pb.store = store.as<rt_photon>();
        pb.keys = keys.as<unsigned long long>();
        pb.store_cap = (uint32_t)std::min<uint64_t>(store_cap, 0xFFFFFFFFull);
        pb.cap = cap;
        pb.cnt = cnt.as<uint32_t>();
        RTB_CUDA(cudaEventRecord(e0, st));
        RTB_CUDA(cudaMemsetAsync(cnt.ptr, 0, 64, st));
        RTB_CUDA(cudaMemsetAsync(perl.ptr, 0, 8ull * nl, st));
        const unsigned blocks = (unsigned)((n + kPB - 1) / kPB);
        k_select<<<blocks, kPB, 0, st>>>(rv, n, seed, dpow.as<float>(), total, sel.as<uint32_t>(),
                                         perl.as<unsigned long long>());
        k_emit<<<blocks, kPB, 0, st>>>(rv, n, seed, dpow.as<float>(), total, sel.as<uint32_t>(),
                                       perl.as<unsigned long long>(), pb);
        RTB_CUDA(cudaGetLastError());
        uint32_t n0 = (uint32_t)n;
        RTB_CUDA(cudaMemcpyAsync(cnt.ptr, &n0, 4, cudaMemcpyHostToDevice, st));
        int cur = 0;
        rays_traced = 0;
        for (uint32_t depth = 0; depth < max_depth; depth++) {
            RTB_CHECK(launch_trace_closest_dev(rv.sv, pb.rays[cur], pb.cnt + cur, cap, pb.hits, RT_TRACE_FAST,
                                               queue.as<uint32_t>(), s->scratch.counters.as<uint32_t>(), st));
            RTB_CUDA(cudaMemsetAsync(pb.cnt + (cur ^ 1), 0, 4, st));
            k_photon_shade<<<cap / kPB + 1, kPB, 0, st>>>(rv, pb, cur, max_depth, rr_depth, seed, flags);
            RTB_CUDA(cudaGetLastError());
            uint32_t hc[4];
            RTB_CUDA(cudaMemcpyAsync(hc, cnt.ptr, 16, cudaMemcpyDeviceToHost, st));
            RTB_CUDA(cudaStreamSynchronize(st));
            rays_traced += hc[cur];
            cur ^= 1;
            if (hc[cur] == 0) break;
        }
        uint32_t hc[4];
        RTB_CUDA(cudaMemcpyAsync(hc, cnt.ptr, 16, cudaMemcpyDeviceToHost, st));
        RTB_CUDA(cudaStreamSynchronize(st));
        stored = hc[2];
        if (stored > store_cap) {  // deterministic: retrace with room for every photon
            store_cap = stored;
            continue;
        }
        // order by (path, depth)
        DevBuf keys_out, idx_in, idx_out, tmp, sorted;
        RTB_CHECK(keys_out.reserve(8 * std::max<uint64_t>(stored, 1)));
        RTB_CHECK(idx_in.reserve(4 * std::max<uint64_t>(stored, 1)));
        RTB_CHECK(idx_out.reserve(4 * std::max<uint64_t>(stored, 1)));
        RTB_CHECK(sorted.reserve(sizeof(rt_photon) * std::max<uint64_t>(stored, 1)));
        if (stored) {
            k_iota<<<(unsigned)((stored + 255) / 256), 256, 0, st>>>(idx_in.as<uint32_t>(), stored);
            size_t tmp_bytes = 0;
            RTB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.as<unsigned long long>(),
                                                     keys_out.as<unsigned long long>(), idx_in.as<uint32_t>(),
                                                     idx_out.as<uint32_t>(), (int)stored, 0, 64, st));
            RTB_CHECK(tmp.reserve(tmp_bytes));
            RTB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tmp_bytes, keys.as<unsigned long long>(),
                                                     keys_out.as<unsigned long long>(), idx_in.as<uint32_t>(),
                                                     idx_out.as<uint32_t>(), (int)stored, 0, 64, st));
            k_gather_photons<<<(unsigned)((stored + 255) / 256), 256, 0, st>>>(store.as<rt_photon>(),
                                                                             idx_out.as<uint32_t>(), stored,
                                                                             sorted.as<rt_photon>());
            RTB_CUDA(cudaGetLastError());
        }
        RTB_CUDA(cudaEventRecord(e1, st));
        RTB_CUDA(cudaEventSynchronize(e1));
        m = new rt_photon_map();
        m->ctx = s->ctx;
        m->n = stored;
        m->photons = std::move(sorted);
        break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!m) return fail(RT_ERR_CAPACITY, "rt_photons_trace: photon store overflow");
    if (stats) {
        stats->emitted = n;
        stats->stored = stored;
        stats->rays = rays_traced;
        stats->ms = ms;
    }
    *out = m;
    return RT_OK;
}

}  // extern "C"
