// Internal declarations shared by the host build code, the kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/rt_b200.h"

namespace rtb {

// ------------------------------------------------------------------ errors

void set_error(const std::string &msg);
int fail(int status, const std::string &msg);
// Records a CUDA error (with location) and returns RT_ERR_CUDA, or RT_OK.
int cuda_status(cudaError_t e, const char *what);

#define RTB_CUDA(call)                                            \
    do {                                                          \
        int rtb_s_ = ::rtb::cuda_status((call), #call);           \
        if (rtb_s_ != RT_OK) return rtb_s_;                       \
    } while (0)

#define RTB_CHECK(expr)                          \
    do {                                         \
        int rtb_s_ = (expr);                     \
        if (rtb_s_ != RT_OK) return rtb_s_;      \
    } while (0)

// Device buffer that remembers its size; grows on demand, never shrinks. Move-only;
// frees its memory when destroyed.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : ptr(o.ptr), bytes(o.bytes)
    {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        if (this != &o) {
            release();
            ptr = o.ptr;
            bytes = o.bytes;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    int reserve(size_t n);  // n bytes at least; contents are not preserved
    int upload(const void *src, size_t n, cudaStream_t s);
    void release();
    template <typename T>
    T *as() const { return static_cast<T *>(ptr); }
};

// Launch sizes derived from occupancy and per-kernel function attributes are properties of
// a device, not of the process: each is cached per CUDA device id.
constexpr int kMaxDevices = 64;
enum DeviceSlot : int {
    SLOT_TRACE_RESIDENT = 0,   // resident blocks of k_trace_closest (SM count x blocks per SM)
    SLOT_SHADOW_RESIDENT = 1,  // resident blocks of the render's k_shadow
    SLOT_GATHER_RESIDENT = 2,  // resident blocks of the render's k_gather
    SLOT_SMEM_ATTRS = 3,       // bit mask of kernels whose dynamic shared-memory limit is raised (SMEM_*)
    SLOT_SM_COUNT = 4,         // multiprocessor count
    SLOT_RETIRE_RESIDENT = 5,  // resident blocks of the render's k_retire
    SLOT_SORT_RESIDENT = 6,    // resident blocks of the render's k_material_sort
    SLOT_MEM_MIB = 7,          // device memory, MiB
    SLOT_COUNT = 8
};
enum SmemAttr : unsigned { SMEM_RENDER_INFER = 1u, SMEM_GUIDE_TRAIN = 2u, SMEM_GUIDE_EVAL = 4u };
// Value of `slot` for the current device; 0 until set_device_slot stored one.
unsigned device_slot(DeviceSlot slot);
void set_device_slot(DeviceSlot slot, unsigned value);
void or_device_slot(DeviceSlot slot, unsigned bits);
// Multiprocessor count of the current device (cached).
unsigned device_sm_count();
// Total memory of the current device in MiB (cached).
unsigned device_mem_mib();

// Error codes written by kernels into the status word (first failure wins).
enum DevError : uint32_t {
    DEV_OK = 0,
    DEV_STACK_OVERFLOW = 1,  // traversal stack would overflow (result of that ray is undefined)
    DEV_STEP_CAP = 2,        // traversal exceeded its step cap
    DEV_QUEUE_OVERFLOW = 3,  // a work queue would overflow
};

// ---------------------------------------------------------- BVH8 layout

// Compressed 8-wide node, 80 bytes (5 x 16 B). Child boxes are quantized to 8 bits per
// axis on a power-of-two grid anchored at `p`; every quantized box contains the child's
// exact box enlarged by the scene's conservative margin, so the float slab test never
// culls a primitive the exact triangle test would hit.
struct alignas(16) Bvh8Node {
    float px, py, pz;      // grid origin
    uint8_t ex, ey, ez;    // biased exponents of the grid step per axis (2^(e-127))
    uint8_t imask;         // bit k: child slot k is an interior node
    uint32_t child_base;   // node index of the first interior child
    uint32_t tri_base;     // record index of the first leaf triangle
    uint8_t meta[8];       // interior: slot's rank among interior children; leaf: (count-1)<<5 | offset
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(Bvh8Node) == 80, "Bvh8Node must be 80 bytes");

// Triangle record in BVH8 leaf order, 48 bytes: the three world-space vertices in the
// reference's vertex order with, in the w lanes, the reference traversal rank, the
// global triangle id and the flags (bit 0: transparent to shadow rays).
struct alignas(16) TriRecord {
    float4 v0;  // w: rank (uint bits)
    float4 v1;  // w: triangle id (uint bits)
    float4 v2;  // w: flags
};

// Analytic shape as the reference stores it: world->object matrix (rows 0..3), radius
// (spheres) and object->world matrix. A plane (kShapePlane) is the unit square [0,1]^2 of its
// object space (shapes/Plane.cu).
constexpr uint32_t kShapePlane = 4u;  // SphereRecord.flags: the record is a Plane
struct alignas(16) SphereRecord {
    float w2o[16];
    float radius;
    uint32_t material;
    int32_t shape_id;
    uint32_t flags;  // bit 0: transparent to shadow rays; bit 1: transparent as added; kShapePlane
    float o2w[16];
};

// One scene of a merged scene (rt_scene_merge): where its BVH8 root lies in the merged node
// array, and its ranges of spheres, emissive triangles and point lights. A path carries the
// index of its scene in the last word of its rays.
constexpr uint32_t kNoRoot = 0xFFFFFFFFu;  // a scene without triangles
struct SubScene {
    uint32_t root;       // node index of its BVH8 root, or kNoRoot
    uint32_t sph0, nsph;  // its spheres
    uint32_t e0, ne;      // its emitters in emit_tri / emit_cdf (the cdf restarts at 0 per scene)
    float etotal;         // sum over its emitters of area * luminance
    uint32_t pl0, npl;    // its point lights
};

// Device view used by the kernels.
struct SceneView {
    const Bvh8Node *nodes;
    const TriRecord *tris;       // leaf order
    const uint32_t *leafpos;     // triangle id -> record index
    const float2 *ref_boxes;     // reference tree boxes, 3 float2 per node (pMin xyz, pMax xyz)
    const uint32_t *ref_sorted;  // sorted position -> triangle id
    const uint32_t *ref_pos;     // triangle id -> sorted position
    const SphereRecord *spheres;
    uint32_t ntri;
    uint32_t nspheres;
    uint32_t nnodes;
    uint32_t root_is_leaf;  // scene with a single leaf (ntri <= 3): node 0 still describes it
    const SubScene *subs;   // merged scene: per-scene roots and ranges (null: one scene, root 0)
    uint32_t nsubs;
};

// ------------------------------------------------------------ host build

struct Bvh8Host {
    std::vector<Bvh8Node> nodes;
    std::vector<uint32_t> leaf_tris;  // record index -> triangle id
};

// Builds the 8-wide BVH over `n` triangles (9 floats each) on the host: PLOC over the
// Morton order `sorted` of the reference-order tree (radius: clusters searched on each side),
// boxes enlarged by `margin` (bvh8_build.cpp).
void build_bvh8(const float *tri9, uint32_t n, float margin, const uint32_t *sorted, uint32_t radius,
                Bvh8Host &out);

// Reference-order tree (cuda_libraries/BVH.cu:314-341): sorted ids, node boxes and
// each triangle's rank in the tree's static traversal order.
struct RefTreeHost {
    std::vector<uint32_t> codes;
    std::vector<uint32_t> sorted;  // sorted position -> triangle id
    std::vector<uint32_t> pos;     // triangle id -> sorted position
    std::vector<float> boxes;      // (2n-1)*6
    std::vector<uint32_t> rank;    // triangle id -> traversal rank
};
void build_ref_tree(const float *tri9, uint32_t n, RefTreeHost &out);

// ---------------------------------------------------------------- kernels

struct TraceScratch {
    DevBuf queue;   // ray indices needing the exact path
    DevBuf counters;  // [0] queue length, [1] status word, [2..] stats
};

int launch_trace_closest(const SceneView &v, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags,
                         uint32_t *queue, uint32_t queue_cap, uint32_t *counters, cudaStream_t s);
// Same with the ray count read on the device (queues built by other kernels); cap bounds it.
int launch_trace_closest_dev(const SceneView &v, const rt_ray *rays, const uint32_t *n_dev, uint32_t cap, rt_hit *hits,
                             uint32_t flags, uint32_t *queue, uint32_t *counters, cudaStream_t s);
// Internal trace flag (above the public RT_TRACE_* bits): trace every ray with tmax = inf,
// as the reference's shadow rays are, whatever tmax the ray carries.
constexpr uint32_t kTraceUnbounded = 0x80000000u;
// Occlusion decided from closest hits: hit and t <= the ray's tmax (Scene::isVisible).
int launch_occlusion_from_hits(const rt_ray *rays, uint64_t n, const rt_hit *hits, void *out, bool bits,
                               cudaStream_t s);
// Any-hit occlusion of n rays: one byte per ray, or (bits) bit i % 32 of word i / 32 (the last
// word's bits past n are 0).
int launch_trace_counts(const SceneView &v, const rt_ray *rays, uint64_t n, uint32_t flags, bool anyhit,
                        uint32_t *counts, uint32_t *counters, cudaStream_t s);
int launch_trace_any(const SceneView &v, const rt_ray *rays, uint64_t n, void *out, bool bits, uint32_t flags,
                     uint32_t *counters, cudaStream_t s);

// Wavefront buffers of rt_render (grown on demand, kept between calls).
struct RenderScratch {
    DevBuf rays[2], st0[2], st1[2], st2[2], hits, srays, scontrib, retire, cnt, gather;
    DevBuf views, view_sample0, view_pixel0;  // the render's views and their prefix sums
    DevBuf perm;  // shading order of the wave (material sort)
    void *host_cnt = nullptr;  // pinned
    double stage_ms[RT_RENDER_STAGES] = {};  // last render's per-stage time (RT_RENDER_STAGE_TIMES)
    void release();
};

}  // namespace rtb

struct rt_scene;
namespace rtb {
// Uploads materials, per-triangle data, emitters and lights when they changed.
int upload_render_data(rt_scene *s);
int upload_textures(rt_scene *s);  // texels and texture table, when textures were added
// Re-derives the shadow-ray transparency of triangle records / spheres from the
// mesh flags and the material table; re-uploads what changed.
int refresh_transparency(rt_scene *s);
// Sets the records' shadow transparency bits on the device from the triangles' flags and
// materials (build_gpu.cu).
int refresh_record_flags(rt_scene *s);
// Builds the reference-order tree and the 8-wide BVH of a scene's triangles on the device,
// byte for byte the host build's (build_gpu.cu); the margin used is returned.
int build_scene_device(rt_scene *s, float margin_out[1]);
}  // namespace rtb

// ------------------------------------------------------------- handles

struct rt_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 0;
    // scratch of the device scene build, kept for the next commit (about 330 bytes per
    // triangle of the largest scene committed): allocating and freeing it per commit cost
    // more than the build
    rtb::DevBuf build[32];
};

struct rt_photon_map {
    rt_context *ctx = nullptr;
    uint64_t n = 0;
    rtb::DevBuf photons;   // rt_photon[n], (path, depth) order
    rtb::DevBuf node_pos;  // float4 per tree slot: xyz, split axis (uint bits)
    rtb::DevBuf node_aux;  // int2 per tree slot: shape id, photon index
    rtb::DevBuf node_pw;   // float4 per tree slot: power rgb, cos(normal, -direction)
    rtb::DevBuf node_dir;  // float4 per tree slot: arrival direction xyz, 0
    bool built = false;
};

struct rt_guide {
    rt_context *ctx = nullptr;
    rt_guide_opts opts{};
    uint64_t step = 0;     // Adam steps taken
    bool trained = false;  // parameters came from training or the caller: rendering samples the guide
    // parameters: FP32 master, Adam moments, last gradient, FP16 shared-memory image
    rtb::DevBuf master, adam_m, adam_v, grad, img;
    // training scratch: transposed activations / gradients, per-chunk weight-gradient
    // partials, scalars ([0] weight mean, [1] loss sum, [2] non-finite flag)
    rtb::DevBuf xt, gt, partial, scal;
    rtb::DevBuf tq, tdir, tpdf, tw;  // batch drawn from the records
    // path-tracer side: decoded mixture per queue slot, training records, the list of records
    // with nonzero weight, the open record of each retiring path, counters ([0] records,
    // [1] nonzero)
    rtb::DevBuf params, recs, nz, retire_rec, rcnt;
    rtb::DevBuf werr;  // evaluation: set when a tensor-core completion wait ran out
    uint32_t rec_cap = 0;
    void *host_scal = nullptr;  // pinned
};

struct rt_scene {
    rt_context *ctx = nullptr;
    // host copies of what was added
    std::vector<float> tri9;           // 9 floats per triangle
    std::vector<uint32_t> tri_material;
    std::vector<int32_t> tri_shape;
    std::vector<uint8_t> tri_transparent;
    std::vector<int32_t> tri_normal_idx;  // 3 per triangle into `normals` (-1: none)
    std::vector<float> normals;
    std::vector<rtb::SphereRecord> spheres;
    bool committed = false;
    uint32_t build_mode = RT_BUILD_DEVICE;
    double build_ms = 0;
    uint64_t nnodes = 0;
    // device
    rtb::DevBuf d_nodes, d_tris, d_leafpos, d_ref_boxes, d_ref_sorted, d_ref_pos, d_spheres;
    rtb::TraceScratch scratch;
    uint64_t last_rays = 0, last_fallback = 0;
    rtb::DevBuf h2d_rays, d2h_hits;  // device staging for the host-buffer entry points
    rtb::DevBuf any_hits;            // closest hits behind rt_trace_any's reference-exact decision
    // merged scene (rt_scene_merge): its scenes' roots and ranges and where each one's
    // triangles start (emitters are gathered per scene at upload)
    bool merged = false;
    std::vector<rtb::SubScene> subs;
    std::vector<uint32_t> sub_tri0;  // nsubs + 1 entries
    rtb::DevBuf d_subs;
    // rendering
    std::vector<rt_material> materials;
    std::vector<float4> plights;  // 2 per light: position, rgb * intensity
    struct PL {
        float r, g, b, i;
    };
    std::vector<PL> plight_rgbi;
    bool render_dirty = true;
    bool has_normals = false;
    uint32_t nemit = 0;
    float emit_total = 0.f;
    rt_photon_map *pmap = nullptr;  // RT_RENDER_PHOTON_MAP gather source
    rt_guide *guide = nullptr;      // RT_RENDER_GUIDE proposal
    int guide_train = 0;            // record training samples while rendering
    uint32_t pm_k = 100;
    // material sort granularity of rt_render (log2 of the chunk; 0: off). BVH-stress render,
    // 1080p x 64 spp, Mrays/s: 1670 off, 1674 / 1754 / 1831 / 1809 / 1799 for 2^6 / 8 / 10 / 12 / 13
    uint32_t sort_log2 = 10;
    float pm_radius = 100.f;
    rtb::DevBuf d_tri_transp, d_mat_transp;  // per-triangle / per-material transparency (record flags)
    // textures: texels (rgb in xyz), per texture (first texel, width, height, 0); texture
    // coordinates, 6 per triangle (empty until rt_scene_set_triangle_uvs; triangles added
    // later get the defaults at upload)
    std::vector<float4> texels;
    std::vector<uint4> tex_info;
    std::vector<float> tri_uv;
    rtb::DevBuf d_texels, d_tex_info, d_tri_uv;
    bool tex_dirty = false;
    rtb::DevBuf d_mats, d_tri_mat, d_tri_shape, d_tri_nidx, d_normals, d_emit_tri, d_emit_cdf, d_plights;
    rtb::RenderScratch rscratch;
    rtb::SceneView view() const;
    uint64_t device_bytes() const;
};
