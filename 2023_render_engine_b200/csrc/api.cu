// C ABI entry points (include/rt_b200.h): contexts, scenes, tracing.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "bvh_common.cuh"
#include "rt_internal.h"

namespace rtb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int status, const std::string &msg)
{
    set_error(msg);
    return status;
}

int cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return RT_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_CUDA;
}

namespace {
std::atomic<unsigned> g_device_slots[kMaxDevices][SLOT_COUNT];

int current_device()
{
    int dev = 0;
    cudaGetDevice(&dev);
    return (dev >= 0 && dev < kMaxDevices) ? dev : 0;
}
}  // namespace

unsigned device_slot(DeviceSlot slot) { return g_device_slots[current_device()][slot].load(); }
void set_device_slot(DeviceSlot slot, unsigned value) { g_device_slots[current_device()][slot].store(value); }
void or_device_slot(DeviceSlot slot, unsigned bits) { g_device_slots[current_device()][slot].fetch_or(bits); }

unsigned device_sm_count()
{
    unsigned n = device_slot(SLOT_SM_COUNT);
    if (!n) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, current_device());
        n = (unsigned)std::max(sms, 1);
        set_device_slot(SLOT_SM_COUNT, n);
    }
    return n;
}

unsigned device_mem_mib()
{
    unsigned m = device_slot(SLOT_MEM_MIB);
    if (!m) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            (void)cudaGetLastError();
            total_b = 0;
        }
        m = (unsigned)std::max<size_t>(total_b >> 20, 1);
        set_device_slot(SLOT_MEM_MIB, m);
    }
    return m;
}

int DevBuf::reserve(size_t n)
{
    if (n <= bytes && ptr) return RT_OK;
    release();
    if (n == 0) return RT_OK;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return cuda_status(e, "cudaMalloc");
    }
    bytes = n;
    return RT_OK;
}

int DevBuf::upload(const void *src, size_t n, cudaStream_t s)
{
    RTB_CHECK(reserve(n));
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, s));
    return RT_OK;
}

void DevBuf::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

// Status word written by kernels -> rt_status.
int check_device_status(uint32_t word)
{
    switch (word) {
    case DEV_OK:
        return RT_OK;
    case DEV_STACK_OVERFLOW:
        return fail(RT_ERR_CAPACITY, "traversal stack overflow: a walk that could not be replayed stopped early");
    case DEV_STEP_CAP:
        return fail(RT_ERR_TIMEOUT, "traversal exceeded its step cap");
    case DEV_QUEUE_OVERFLOW:
        return fail(RT_ERR_CAPACITY, "exact-traversal queue overflow");
    default:
        return fail(RT_ERR_CUDA, "unknown device status");
    }
}

}  // namespace rtb

using namespace rtb;

rtb::SceneView rt_scene::view() const
{
    SceneView v{};
    v.nodes = d_nodes.as<Bvh8Node>();
    v.tris = d_tris.as<TriRecord>();
    v.leafpos = d_leafpos.as<uint32_t>();
    v.ref_boxes = d_ref_boxes.as<float2>();
    v.ref_sorted = d_ref_sorted.as<uint32_t>();
    v.ref_pos = d_ref_pos.as<uint32_t>();
    v.spheres = d_spheres.as<SphereRecord>();
    v.ntri = (uint32_t)(tri9.size() / 9);
    v.nspheres = (uint32_t)spheres.size();
    v.nnodes = (uint32_t)nnodes;
    v.subs = merged ? d_subs.as<SubScene>() : nullptr;
    v.nsubs = merged ? (uint32_t)subs.size() : 0u;
    return v;
}

uint64_t rt_scene::device_bytes() const
{
    return d_nodes.bytes + d_tris.bytes + d_leafpos.bytes + d_ref_boxes.bytes + d_ref_sorted.bytes + d_ref_pos.bytes +
           d_spheres.bytes + scratch.queue.bytes + scratch.counters.bytes + d_tri_transp.bytes + d_mat_transp.bytes;
}

extern "C" {

int rt_abi_version(void) { return RT_B200_ABI_VERSION; }

int rt_last_error(char *buf, size_t len)
{
    if (!buf || len == 0) return RT_ERR_INVALID;
    size_t n = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), n);
    buf[n] = 0;
    return RT_OK;
}

int rt_context_create(int device, rt_context **out)
{
    if (!out) return fail(RT_ERR_INVALID, "rt_context_create: out is null");
    int count = 0;
    RTB_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(RT_ERR_INVALID, "rt_context_create: no such device");
    RTB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    RTB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(RT_ERR_UNSUPPORTED, "rt_context_create: sm_100a (B200) required");
    rt_context *c = new rt_context();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_status(e, "cudaStreamCreate");
    }
    c->own_stream = true;
    *out = c;
    return RT_OK;
}

int rt_context_destroy(rt_context *ctx)
{
    if (!ctx) return RT_OK;
    cudaSetDevice(ctx->device);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return RT_OK;
}

int rt_context_set_stream(rt_context *ctx, void *stream)
{
    if (!ctx) return fail(RT_ERR_INVALID, "rt_context_set_stream: null context");
    if (ctx->own_stream && ctx->stream) {
        RTB_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaStreamDestroy(ctx->stream);
    }
    ctx->stream = static_cast<cudaStream_t>(stream);
    ctx->own_stream = false;
    return RT_OK;
}

int rt_context_synchronize(rt_context *ctx)
{
    if (!ctx) return fail(RT_ERR_INVALID, "rt_context_synchronize: null context");
    RTB_CUDA(cudaSetDevice(ctx->device));
    RTB_CUDA(cudaStreamSynchronize(ctx->stream));
    return RT_OK;
}

int rt_scene_create(rt_context *ctx, rt_scene **out)
{
    if (!ctx || !out) return fail(RT_ERR_INVALID, "rt_scene_create: null argument");
    rt_scene *s = new rt_scene();
    s->ctx = ctx;
    *out = s;
    return RT_OK;
}

int rt_scene_destroy(rt_scene *s)
{
    if (!s) return RT_OK;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    for (DevBuf *b : {&s->d_nodes, &s->d_tris, &s->d_leafpos, &s->d_ref_boxes, &s->d_ref_sorted, &s->d_ref_pos,
                      &s->d_spheres, &s->scratch.queue, &s->scratch.counters, &s->h2d_rays, &s->d2h_hits, &s->d_mats,
                      &s->d_tri_mat, &s->d_tri_shape, &s->d_tri_nidx, &s->d_normals, &s->d_emit_tri, &s->d_emit_cdf, &s->d_plights})
        b->release();
    s->rscratch.release();
    delete s;
    return RT_OK;
}

int rt_scene_add_mesh(rt_scene *s, const float *xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri,
                      const float *normals, uint32_t nn, const uint32_t *nidx, uint32_t material, int32_t shape_id,
                      int transparent, uint32_t *first_tri)
{
    if (!s || (!xyz && nv) || (!idx && ntri)) return fail(RT_ERR_INVALID, "rt_scene_add_mesh: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_add_mesh: not available on a merged scene");
    if ((normals == nullptr) != (nidx == nullptr)) return fail(RT_ERR_INVALID, "rt_scene_add_mesh: normals need nidx");
    uint64_t base = s->tri9.size() / 9;
    if (base + ntri >= 0x40000000ull) return fail(RT_ERR_CAPACITY, "rt_scene_add_mesh: more than 2^30 triangles");
    for (uint64_t i = 0; i < 3ull * ntri; i++) {
        if (idx[i] >= nv) return fail(RT_ERR_INVALID, "rt_scene_add_mesh: vertex index out of range");
        if (nidx && nidx[i] >= nn) return fail(RT_ERR_INVALID, "rt_scene_add_mesh: normal index out of range");
    }
    uint32_t nbase = (uint32_t)(s->normals.size() / 3);
    if (normals) s->normals.insert(s->normals.end(), normals, normals + 3ull * nn);
    s->tri9.reserve(s->tri9.size() + 9ull * ntri);
    for (uint32_t t = 0; t < ntri; t++) {
        for (int k = 0; k < 3; k++) {
            const float *p = xyz + 3ull * idx[3ull * t + k];
            s->tri9.push_back(p[0]);
            s->tri9.push_back(p[1]);
            s->tri9.push_back(p[2]);
            s->tri_normal_idx.push_back(nidx ? (int32_t)(nbase + nidx[3ull * t + k]) : -1);
        }
        s->tri_material.push_back(material);
        s->tri_shape.push_back(shape_id);
        s->tri_transparent.push_back(transparent ? 1 : 0);
    }
    if (first_tri) *first_tri = (uint32_t)base;
    s->committed = false;
    return RT_OK;
}

int rt_scene_add_sphere(rt_scene *s, const float o2w[16], const float w2o[16], float radius, uint32_t material,
                        int32_t shape_id, int transparent, uint32_t *index)
{
    if (!s || !o2w || !w2o) return fail(RT_ERR_INVALID, "rt_scene_add_sphere: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_add_sphere: not available on a merged scene");
    if (!(radius > 0)) return fail(RT_ERR_INVALID, "rt_scene_add_sphere: radius must be positive");
    SphereRecord r{};
    std::memcpy(r.w2o, w2o, sizeof(r.w2o));
    std::memcpy(r.o2w, o2w, sizeof(r.o2w));
    r.radius = radius;
    r.material = material;
    r.shape_id = shape_id;
    r.flags = transparent ? 3u : 0u;  // bit 1: requested at add time, bit 0: effective
    if (index) *index = (uint32_t)s->spheres.size();
    s->spheres.push_back(r);
    s->committed = false;
    return RT_OK;
}

int rt_scene_add_plane(rt_scene *s, const float o2w[16], const float w2o[16], uint32_t material, int32_t shape_id,
                       int transparent, uint32_t *index)
{
    if (!s || !o2w || !w2o) return fail(RT_ERR_INVALID, "rt_scene_add_plane: null argument");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_add_plane: not available on a merged scene");
    SphereRecord r{};
    std::memcpy(r.w2o, w2o, sizeof(r.w2o));
    std::memcpy(r.o2w, o2w, sizeof(r.o2w));
    r.radius = 0.f;
    r.material = material;
    r.shape_id = shape_id;
    r.flags = kShapePlane | (transparent ? 3u : 0u);
    if (index) *index = (uint32_t)s->spheres.size();
    s->spheres.push_back(r);
    s->committed = false;
    return RT_OK;
}

int rt_scene_set_build(rt_scene *s, uint32_t mode)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_scene_set_build: null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_set_build: not available on a merged scene");
    if (mode != RT_BUILD_DEVICE && mode != RT_BUILD_HOST) return fail(RT_ERR_INVALID, "rt_scene_set_build: bad mode");
    s->build_mode = mode;
    return RT_OK;
}

int rt_scene_commit(rt_scene *s)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_scene_commit: null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_scene_commit: not available on a merged scene");
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    auto t0 = std::chrono::steady_clock::now();
    const uint32_t n = (uint32_t)(s->tri9.size() / 9);
    if (n > 0 && s->build_mode == RT_BUILD_DEVICE) {
        float margin = 0.f;
        RTB_CHECK(build_scene_device(s, &margin));
    } else {
        // conservative margin: 1e-5 of the largest coordinate magnitude
        float maxabs = 0.f;
        for (float x : s->tri9) maxabs = std::max(maxabs, std::fabs(x));
        const float margin = std::max(1e-5f * maxabs, 1e-30f);
        Bvh8Host bvh;
        RefTreeHost ref;
        build_ref_tree(s->tri9.data(), n, ref);
        build_bvh8(s->tri9.data(), n, margin, ref.sorted.data(), kPlocRadius, bvh);
        std::vector<TriRecord> recs(bvh.leaf_tris.size());
        std::vector<uint32_t> leafpos(n, 0);
        for (size_t r = 0; r < bvh.leaf_tris.size(); r++) {
            uint32_t id = bvh.leaf_tris[r];
            const float *p = s->tri9.data() + 9ull * id;
            TriRecord &tr = recs[r];
            uint32_t rank = ref.rank[id], flags = s->tri_transparent[id];
            tr.v0 = make_float4(p[0], p[1], p[2], 0.f);
            tr.v1 = make_float4(p[3], p[4], p[5], 0.f);
            tr.v2 = make_float4(p[6], p[7], p[8], 0.f);
            std::memcpy(&tr.v0.w, &rank, 4);
            std::memcpy(&tr.v1.w, &id, 4);
            std::memcpy(&tr.v2.w, &flags, 4);
            leafpos[id] = (uint32_t)r;
        }
        if (bvh.nodes.empty()) {
            bvh.nodes.resize(1);
            std::memset(bvh.nodes.data(), 0, sizeof(Bvh8Node));
            std::memset(bvh.nodes[0].meta, 0xFF, 8);
        }
        s->nnodes = bvh.nodes.size();
        RTB_CHECK(s->d_nodes.upload(bvh.nodes.data(), bvh.nodes.size() * sizeof(Bvh8Node), st));
        RTB_CHECK(s->d_tris.upload(recs.data(), recs.size() * sizeof(TriRecord), st));
        RTB_CHECK(s->d_leafpos.upload(leafpos.data(), leafpos.size() * 4, st));
        RTB_CHECK(s->d_ref_boxes.upload(ref.boxes.data(), ref.boxes.size() * 4, st));
        RTB_CHECK(s->d_ref_sorted.upload(ref.sorted.data(), ref.sorted.size() * 4, st));
        RTB_CHECK(s->d_ref_pos.upload(ref.pos.data(), ref.pos.size() * 4, st));
    }
    s->render_dirty = true;
    RTB_CHECK(s->d_spheres.upload(s->spheres.data(), s->spheres.size() * sizeof(SphereRecord), st));
    RTB_CHECK(s->scratch.counters.reserve(64));
    RTB_CHECK(refresh_transparency(s));
    RTB_CUDA(cudaStreamSynchronize(st));
    s->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    s->committed = true;
    return RT_OK;
}

int rt_scene_export_bvh(rt_scene *s, void *nodes, void *records, float *ref_boxes, uint64_t *nnodes,
                        uint64_t *nrecords, uint64_t *nref_nodes)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_scene_export_bvh: null scene");
    if (!s->committed) return fail(RT_ERR_STATE, "rt_scene_export_bvh: scene not committed");
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    const uint64_t n = s->tri9.size() / 9;
    const uint64_t nref = n ? 2 * n - 1 : 0;
    if (nnodes) *nnodes = s->nnodes;
    if (nrecords) *nrecords = n;
    if (nref_nodes) *nref_nodes = nref;
    if (nodes && s->nnodes)
        RTB_CUDA(cudaMemcpyAsync(nodes, s->d_nodes.ptr, s->nnodes * sizeof(Bvh8Node), cudaMemcpyDeviceToHost, st));
    if (records && n) RTB_CUDA(cudaMemcpyAsync(records, s->d_tris.ptr, n * sizeof(TriRecord), cudaMemcpyDeviceToHost, st));
    if (ref_boxes && nref)
        RTB_CUDA(cudaMemcpyAsync(ref_boxes, s->d_ref_boxes.ptr, nref * 24, cudaMemcpyDeviceToHost, st));
    RTB_CUDA(cudaStreamSynchronize(st));
    return RT_OK;
}

int rt_scene_stats_get(rt_scene *s, rt_scene_stats *out)
{
    if (!s || !out) return fail(RT_ERR_INVALID, "rt_scene_stats_get: null argument");
    out->triangles = s->tri9.size() / 9;
    out->spheres = s->spheres.size();
    out->bvh8_nodes = s->nnodes;
    out->bvh8_leaf_triangles = s->committed ? s->tri9.size() / 9 : 0;
    out->device_bytes = s->device_bytes();
    out->build_ms = s->build_ms;
    return RT_OK;
}

static int trace_common(rt_scene *s, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_trace_closest: null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_trace_closest: not available on a merged scene");
    if (!s->committed) return fail(RT_ERR_STATE, "rt_trace_closest: scene not committed");
    if (n && (!rays || !hits)) return fail(RT_ERR_INVALID, "rt_trace_closest: null buffer");
    if (n >= 0x80000000ull) return fail(RT_ERR_INVALID, "rt_trace_closest: at most 2^31-1 rays per call");
    if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u)
        return fail(RT_ERR_INVALID, "rt_trace_closest: buffers must be 16-byte aligned");
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    RTB_CHECK(s->scratch.queue.reserve(std::max<uint64_t>(n, 1) * 4));
    RTB_CHECK(launch_trace_closest(s->view(), rays, n, hits, flags, s->scratch.queue.as<uint32_t>(), (uint32_t)n,
                                   s->scratch.counters.as<uint32_t>(), s->ctx->stream));
    return RT_OK;
}

static int finish_trace(rt_scene *s, uint64_t n)
{
    s->last_rays = n;
    s->last_fallback = 0;
    if (n == 0) return RT_OK;  // nothing launched: the counters still hold an earlier call's
    uint32_t c[4] = {0, 0, 0, 0};
    RTB_CUDA(cudaMemcpyAsync(c, s->scratch.counters.ptr, sizeof(c), cudaMemcpyDeviceToHost, s->ctx->stream));
    RTB_CUDA(cudaStreamSynchronize(s->ctx->stream));
    s->last_fallback = c[0];
    return check_device_status(c[1]);
}

int rt_trace_closest(rt_scene *s, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags)
{
    RTB_CHECK(trace_common(s, rays, n, hits, flags));
    return finish_trace(s, n);
}

int rt_trace_closest_host(rt_scene *s, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_trace_closest_host: null scene");
    if (n && (!rays || !hits)) return fail(RT_ERR_INVALID, "rt_trace_closest_host: null buffer");
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    RTB_CHECK(s->h2d_rays.reserve(std::max<uint64_t>(n, 1) * sizeof(rt_ray)));
    RTB_CHECK(s->d2h_hits.reserve(std::max<uint64_t>(n, 1) * sizeof(rt_hit)));
    RTB_CUDA(cudaMemcpyAsync(s->h2d_rays.ptr, rays, n * sizeof(rt_ray), cudaMemcpyHostToDevice, st));
    RTB_CHECK(trace_common(s, s->h2d_rays.as<rt_ray>(), n, s->d2h_hits.as<rt_hit>(), flags));
    RTB_CUDA(cudaMemcpyAsync(hits, s->d2h_hits.ptr, n * sizeof(rt_hit), cudaMemcpyDeviceToHost, st));
    return finish_trace(s, n);
}

static int trace_any_common(rt_scene *s, const rt_ray *rays, uint64_t n, void *out, bool bits, uint32_t flags,
                            const char *who)
{
    if (!s) return fail(RT_ERR_INVALID, std::string(who) + ": null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, std::string(who) + ": not available on a merged scene");
    if (!s->committed) return fail(RT_ERR_STATE, std::string(who) + ": scene not committed");
    if (n && (!rays || !out)) return fail(RT_ERR_INVALID, std::string(who) + ": null buffer");
    if (n >= 0x80000000ull) return fail(RT_ERR_INVALID, std::string(who) + ": at most 2^31-1 rays per call");
    if (reinterpret_cast<uintptr_t>(rays) & 15u)
        return fail(RT_ERR_INVALID, std::string(who) + ": rays must be 16-byte aligned");
    if (bits && (reinterpret_cast<uintptr_t>(out) & 3u))
        return fail(RT_ERR_INVALID, std::string(who) + ": the bit mask must be 4-byte aligned");
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    if (flags & RT_TRACE_FAST) {
        RTB_CHECK(launch_trace_any(s->view(), rays, n, out, bits, flags, s->scratch.counters.as<uint32_t>(), st));
    } else {
        // the reference's decision: its closest hit along the unbounded ray, then t <= tmax
        RTB_CHECK(s->scratch.queue.reserve(n * 4));
        RTB_CHECK(s->any_hits.reserve(n * sizeof(rt_hit)));
        RTB_CHECK(launch_trace_closest(s->view(), rays, n, s->any_hits.as<rt_hit>(),
                                       (flags & RT_TRACE_SHADOW) | kTraceUnbounded, s->scratch.queue.as<uint32_t>(),
                                       (uint32_t)n, s->scratch.counters.as<uint32_t>(), st));
        RTB_CHECK(launch_occlusion_from_hits(rays, n, s->any_hits.as<rt_hit>(), out, bits, st));
    }
    uint32_t c[4] = {0, 0, 0, 0};
    RTB_CUDA(cudaMemcpyAsync(c, s->scratch.counters.ptr, sizeof(c), cudaMemcpyDeviceToHost, s->ctx->stream));
    RTB_CUDA(cudaStreamSynchronize(s->ctx->stream));
    return check_device_status(c[1]);
}

int rt_trace_any(rt_scene *s, const rt_ray *rays, uint64_t n, uint8_t *occluded, uint32_t flags)
{
    return trace_any_common(s, rays, n, occluded, false, flags, "rt_trace_any");
}

int rt_trace_any_bits(rt_scene *s, const rt_ray *rays, uint64_t n, uint32_t *occluded_bits, uint32_t flags)
{
    return trace_any_common(s, rays, n, occluded_bits, true, flags, "rt_trace_any_bits");
}

int rt_trace_counts(rt_scene *s, const rt_ray *rays, uint64_t n, uint32_t flags, uint32_t *counts)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_trace_counts: null scene");
    if (s->merged) return fail(RT_ERR_UNSUPPORTED, "rt_trace_counts: not available on a merged scene");
    if (!s->committed) return fail(RT_ERR_STATE, "rt_trace_counts: scene not committed");
    if (n && (!rays || !counts)) return fail(RT_ERR_INVALID, "rt_trace_counts: null buffer");
    if (n >= 0x80000000ull) return fail(RT_ERR_INVALID, "rt_trace_counts: at most 2^31-1 rays per call");
    if ((reinterpret_cast<uintptr_t>(rays) & 15u) || (reinterpret_cast<uintptr_t>(counts) & 7u))
        return fail(RT_ERR_INVALID, "rt_trace_counts: rays must be 16-byte and counts 8-byte aligned");
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaSetDevice(s->ctx->device));
    cudaStream_t st = s->ctx->stream;
    RTB_CHECK(launch_trace_counts(s->view(), rays, n, flags & RT_TRACE_SHADOW, (flags & RT_TRACE_COUNT_ANY) != 0,
                                  counts, s->scratch.counters.as<uint32_t>(), st));
    uint32_t c[4] = {0, 0, 0, 0};
    RTB_CUDA(cudaMemcpyAsync(c, s->scratch.counters.ptr, sizeof(c), cudaMemcpyDeviceToHost, st));
    RTB_CUDA(cudaStreamSynchronize(st));
    if (c[1] == DEV_STACK_OVERFLOW)
        return fail(RT_ERR_CAPACITY, "rt_trace_counts: a ray's walk ran out of stack; its counts stop there");
    return check_device_status(c[1]);
}

int rt_trace_stats_get(rt_scene *s, rt_trace_stats *out)
{
    if (!s || !out) return fail(RT_ERR_INVALID, "rt_trace_stats_get: null argument");
    out->rays = s->last_rays;
    out->exact_fallback_rays = s->last_fallback;
    return RT_OK;
}

}  // extern "C"
