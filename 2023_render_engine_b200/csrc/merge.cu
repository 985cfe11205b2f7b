// rt_scene_merge: several committed scenes rendered as one wavefront (new in this build; the
// reference renders one scene per PathTracerIntegrator::render call,
// integration/PathTracerIntegrator.cu:140-210).
//
// The merged scene keeps every scene's own 8-wide BVH: the node, triangle-record and leaf
// tables are concatenated on the device and their internal indices moved by the offsets of
// the scenes before (child and record bases of the nodes, triangle ids of the records, record
// positions of the triangles). A path carries its scene's index in its rays, and traversal
// starts at that scene's root; spheres, emitters and point lights are looked up in the
// scene's own ranges. Materials, textures and per-triangle data are concatenated with their
// ids moved the same way, so the shading kernels run unchanged on global ids.
#include <algorithm>

#include "rt_internal.h"

namespace rtb {
namespace {

constexpr int kT = 256;

__global__ void k_rebase_nodes(Bvh8Node *__restrict__ nodes, uint64_t n, uint32_t node_off, uint32_t rec_off)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    nodes[i].child_base += node_off;
    nodes[i].tri_base += rec_off;
}

__global__ void k_rebase_records(TriRecord *__restrict__ recs, uint64_t n, uint32_t tri_off)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    recs[i].v1.w = __uint_as_float(__float_as_uint(recs[i].v1.w) + tri_off);  // triangle id
}

__global__ void k_add_u32(uint32_t *__restrict__ a, uint64_t n, uint32_t off)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] += off;
}

unsigned blocks(uint64_t n) { return (unsigned)std::max<uint64_t>(1, (n + kT - 1) / kT); }

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" int rt_scene_merge(rt_context *ctx, rt_scene *const *scenes, uint32_t n, rt_scene **out)
{
    if (!ctx || !scenes || !out || n == 0) return fail(RT_ERR_INVALID, "rt_scene_merge: null argument");
    if (n > 256) return fail(RT_ERR_INVALID, "rt_scene_merge: at most 256 scenes");
    uint64_t ntri = 0, nnodes = 0;
    for (uint32_t k = 0; k < n; k++) {
        const rt_scene *s = scenes[k];
        if (!s) return fail(RT_ERR_INVALID, "rt_scene_merge: null scene");
        if (s->ctx != ctx) return fail(RT_ERR_INVALID, "rt_scene_merge: scenes of another context");
        if (!s->committed) return fail(RT_ERR_STATE, "rt_scene_merge: every scene must be committed");
        if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_merge: a merged scene cannot be merged again");
        ntri += s->tri9.size() / 9;
        nnodes += s->nnodes;
    }
    if (ntri >= 0x40000000ull) return fail(RT_ERR_CAPACITY, "rt_scene_merge: too many triangles");
    RTB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    rt_scene *m = new rt_scene();
    m->ctx = ctx;
    m->merged = true;
    auto cleanup = [&](int rc) {
        delete m;
        return rc;
    };
    int rc = RT_OK;
    if ((rc = m->d_nodes.reserve(std::max<uint64_t>(nnodes, 1) * sizeof(Bvh8Node))) != RT_OK) return cleanup(rc);
    if ((rc = m->d_tris.reserve(std::max<uint64_t>(ntri, 1) * sizeof(TriRecord))) != RT_OK) return cleanup(rc);
    if ((rc = m->d_leafpos.reserve(std::max<uint64_t>(ntri, 1) * 4)) != RT_OK) return cleanup(rc);
    bool any_uv = false;
    for (uint32_t k = 0; k < n; k++) any_uv |= !scenes[k]->tri_uv.empty();
    uint32_t tri_off = 0, node_off = 0, mat_off = 0, tex_off = 0, texel_off = 0, normal_off = 0;
    for (uint32_t k = 0; k < n; k++) {
        const rt_scene *s = scenes[k];
        const uint32_t nt = (uint32_t)(s->tri9.size() / 9), nn = (uint32_t)s->nnodes;
        SubScene sub{};
        sub.root = nt ? node_off : kNoRoot;
        sub.sph0 = (uint32_t)m->spheres.size();
        sub.nsph = (uint32_t)s->spheres.size();
        sub.pl0 = (uint32_t)(m->plights.size() / 2);
        sub.npl = (uint32_t)(s->plights.size() / 2);
        m->subs.push_back(sub);
        m->sub_tri0.push_back(tri_off);
        // device: this scene's BVH8, records and leaf positions, moved by the offsets before it
        if (nt) {
            Bvh8Node *dn = m->d_nodes.as<Bvh8Node>() + node_off;
            TriRecord *dr = m->d_tris.as<TriRecord>() + tri_off;
            uint32_t *dl = m->d_leafpos.as<uint32_t>() + tri_off;
            RTB_CUDA(cudaMemcpyAsync(dn, s->d_nodes.ptr, (uint64_t)nn * sizeof(Bvh8Node), cudaMemcpyDeviceToDevice, st));
            RTB_CUDA(cudaMemcpyAsync(dr, s->d_tris.ptr, (uint64_t)nt * sizeof(TriRecord), cudaMemcpyDeviceToDevice, st));
            RTB_CUDA(cudaMemcpyAsync(dl, s->d_leafpos.ptr, (uint64_t)nt * 4, cudaMemcpyDeviceToDevice, st));
            k_rebase_nodes<<<blocks(nn), kT, 0, st>>>(dn, nn, node_off, tri_off);
            k_rebase_records<<<blocks(nt), kT, 0, st>>>(dr, nt, tri_off);
            k_add_u32<<<blocks(nt), kT, 0, st>>>(dl, nt, tri_off);
            RTB_CUDA(cudaGetLastError());
        }
        // host: per-triangle data, materials, spheres, lights and textures with their ids moved
        m->tri9.insert(m->tri9.end(), s->tri9.begin(), s->tri9.end());
        for (uint32_t t = 0; t < nt; t++) m->tri_material.push_back(s->tri_material[t] + mat_off);
        m->tri_shape.insert(m->tri_shape.end(), s->tri_shape.begin(), s->tri_shape.end());
        m->tri_transparent.insert(m->tri_transparent.end(), s->tri_transparent.begin(), s->tri_transparent.end());
        for (int32_t x : s->tri_normal_idx) m->tri_normal_idx.push_back(x >= 0 ? x + (int32_t)normal_off : x);
        m->normals.insert(m->normals.end(), s->normals.begin(), s->normals.end());
        for (rt_material mt : s->materials) {
            if (mt.texture) mt.texture += tex_off;
            m->materials.push_back(mt);
        }
        for (SphereRecord sp : s->spheres) {
            sp.material += mat_off;
            m->spheres.push_back(sp);
        }
        m->plights.insert(m->plights.end(), s->plights.begin(), s->plights.end());
        m->plight_rgbi.insert(m->plight_rgbi.end(), s->plight_rgbi.begin(), s->plight_rgbi.end());
        m->texels.insert(m->texels.end(), s->texels.begin(), s->texels.end());
        for (uint4 ti : s->tex_info) {
            ti.x += texel_off;
            m->tex_info.push_back(ti);
        }
        if (any_uv) {
            if (s->tri_uv.size() >= 6ull * nt) {
                m->tri_uv.insert(m->tri_uv.end(), s->tri_uv.begin(), s->tri_uv.begin() + 6ull * nt);
            } else {
                for (uint32_t t = 0; t < nt; t++) m->tri_uv.insert(m->tri_uv.end(), {0.f, 0.f, 1.f, 0.f, 1.f, 1.f});
            }
        }
        tri_off += nt;
        node_off += nn;
        mat_off += (uint32_t)s->materials.size();
        tex_off += (uint32_t)s->tex_info.size();
        texel_off += (uint32_t)s->texels.size();
        normal_off += (uint32_t)(s->normals.size() / 3);
    }
    m->sub_tri0.push_back(tri_off);
    m->nnodes = nnodes;
    if (!m->spheres.empty())
        if ((rc = m->d_spheres.upload(m->spheres.data(), m->spheres.size() * sizeof(SphereRecord), st)) != RT_OK)
            return cleanup(rc);
    if ((rc = m->d_subs.upload(m->subs.data(), m->subs.size() * sizeof(SubScene), st)) != RT_OK) return cleanup(rc);
    if ((rc = m->scratch.counters.reserve(64)) != RT_OK) return cleanup(rc);
    m->has_normals = false;
    m->tex_dirty = true;
    m->render_dirty = true;
    m->committed = true;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cleanup(cuda_status(e, "rt_scene_merge"));
    *out = m;
    return RT_OK;
}
