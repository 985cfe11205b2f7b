// Closest-hit and occlusion traversal of the compressed 8-wide BVH (sm_100a).
//
// One thread per ray. A node is 80 bytes (five 16-byte read-only loads); its eight
// quantized child boxes are slab-tested against the ray, hit leaves are intersected at
// once with the reference's watertight arithmetic (exact_math.cuh), hit interior
// children are sorted near-to-far and the far ones pushed on a per-thread stack.
//
// Reference parity (rt_trace_closest without RT_TRACE_FAST): the reference traversal
// (BVH::intersectRay, cuda_libraries/BVH.cu:355-448) returns, among the triangles it
// reaches, the last one in its static order that lowers its running offset and passes
// the error-bound test (Triangle.cu:569-593). That equals "smallest offset, ties to the
// highest static rank" — what the kernel computes — unless (a) the winner is not
// reached because an ancestor box of the reference tree misses the ray, or (b) some
// triangle with a smaller offset fails the error-bound test after lowering the running
// offset. The kernel proves (a) cannot happen with one slab test on the winner's own
// box (float rounding is monotonic, so every ancestor box passes when the winner's box
// does, for rays with tmax = inf and no zero direction component) and detects (b); the
// remaining rays are queued for a replay of the reference traversal itself
// (k_trace_exact).
#include <algorithm>

#include "traverse.cuh"

namespace rtb {

namespace {

constexpr int kBlock = 128;

// Decides, for a finished ray, whether the kernel's answer provably equals the reference's
// (see the file comment) and writes the hit, or queues the ray for k_trace_exact.
// A merged scene (rt_scene_merge) has no reference-order tree: its rays are traced in the fast
// mode, and a ray whose walk ran out of stack keeps the hit found so far (status word set).
__device__ __forceinline__ void closest_epilogue(const SceneView &v, uint64_t i, uint32_t sub, const Trav &T,
                                                 uint32_t flags, rt_hit *__restrict__ hits,
                                                 uint32_t *__restrict__ queue, uint32_t queue_cap,
                                                 uint32_t *__restrict__ counters)
{
    const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
    const Best &best = T.best;
    const float ox = T.w.ox, oy = T.w.oy, oz = T.w.oz, tmax = T.w.tmax;
    bool exact_needed = false, replay = false;
    if (!T.ok) {
        // the walk ran out of stack or steps: the reference-order replay gives the exact answer
        // (its own overflow is reported by k_trace_exact); a merged scene has no reference tree,
        // so there the status word reports that the hit found so far is kept
        exact_needed = replay = v.subs == nullptr;
        if (v.subs) atomicCAS(counters + 1, 0u, (uint32_t)DEV_STACK_OVERFLOW);
    } else if (!(flags & RT_TRACE_FAST) && best.prim >= 0) {
        if (best.minblock < best.t) {
            exact_needed = replay = true;
        } else if (!(tmax == INFINITY) || T.dx == 0.f || T.dy == 0.f || T.dz == 0.f) {
            exact_needed = true;  // ancestor walk in k_trace_exact
        } else {
            const float4 *p = reinterpret_cast<const float4 *>(v.tris + v.leafpos[best.prim]);
            float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
            float lx = fminf(fminf(a.x, b.x), c.x), ly = fminf(fminf(a.y, b.y), c.y), lz = fminf(fminf(a.z, b.z), c.z);
            float hx = fmaxf(fmaxf(a.x, b.x), c.x), hy = fmaxf(fmaxf(a.y, b.y), c.y), hz = fmaxf(fmaxf(a.z, b.z), c.z);
            float ix = fdiv(1.0f, T.dx), iy = fdiv(1.0f, T.dy), iz = fdiv(1.0f, T.dz);
            if (!ref_box_test(lx, ly, lz, hx, hy, hz, ox, oy, oz, ix, iy, iz, tmax)) exact_needed = true;
        }
    }
    if (exact_needed) {
        uint32_t slot = atomicAdd(counters, 1u);
        if (slot < queue_cap) {
            queue[slot] = (uint32_t)i | (replay ? kQueueBlocker : 0u);
            hits[i] = rt_hit{best.t, best.prim, best.b1, best.b2};
            return;
        }
        atomicCAS(counters + 1, 0u, (uint32_t)DEV_QUEUE_OVERFLOW);
    }
    float t = best.prim >= 0 ? best.t : INFINITY;
    int32_t prim = best.prim;
    float b1 = best.b1, b2 = best.b2;
    intersect_spheres(v, sub, ox, oy, oz, T.dx, T.dy, T.dz, tmax, shadow, t, prim, b1, b2);
    reinterpret_cast<float4 *>(hits)[i] = make_float4(t, __int_as_float(prim), b1, b2);
}

// Scene index a ray carries in its last word (merged scenes only; 0 otherwise).
__device__ __forceinline__ uint32_t ray_scene(const SceneView &v, const rt_ray *rays, uint64_t i)
{
    return v.subs ? __float_as_uint(__ldg(reinterpret_cast<const float *>(rays) + 8 * i + 7)) : 0u;
}

// Persistent closest-hit kernel: warps fetch rays from counters[3] until all n are done.
__global__ void __launch_bounds__(kBlock, RTB_TRAV_MIN_BLOCKS) k_trace_closest(SceneView v, const rt_ray *__restrict__ rays, uint64_t n,
                                                          const uint32_t *__restrict__ n_dev, rt_hit *__restrict__ hits,
                                                          uint32_t flags, uint32_t *__restrict__ queue,
                                                          uint32_t queue_cap, uint32_t *__restrict__ counters)
{
    if (n_dev) n = min((uint64_t)*n_dev, n);
    const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
    persistent_traverse(
        v, (uint32_t)n, counters + 3, false,
        [&](uint32_t i, Trav &T) {
            float4 ra, rb;
            load_ray(rays, i, ra, rb);
            const uint32_t root = scene_root(v, v.subs ? __float_as_uint(rb.w) : 0u);
            trav_init(T, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, (flags & kTraceUnbounded) ? INFINITY : ra.w, root);
            T.shadow = shadow;
        },
        [&](uint32_t i, Trav &T) {
            closest_epilogue(v, i, ray_scene(v, rays, i), T, flags, hits, queue, queue_cap, counters);
        });
}

// Traversal work per ray (rt_trace_counts): the persistent walk of k_trace_closest without its
// exactness checks (closest hit) or the any-hit walk of the renderer's shadow rays, writing for
// ray i the BVH8 nodes it visited and the triangle records it tested.
__global__ void __launch_bounds__(kBlock, RTB_TRAV_MIN_BLOCKS) k_trace_counts(SceneView v, const rt_ray *__restrict__ rays,
                                                                             uint64_t n, uint32_t flags, bool anyhit,
                                                                             uint2 *__restrict__ counts,
                                                                             uint32_t *__restrict__ counters)
{
    const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
    persistent_traverse<true>(
        v, (uint32_t)n, counters + 3, anyhit,
        [&](uint32_t i, Trav &T) {
            float4 ra, rb;
            load_ray(rays, i, ra, rb);
            trav_init(T, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w, scene_root(v, 0));
            T.shadow = shadow;
        },
        [&](uint32_t i, Trav &T) {
            if (!T.ok)
                atomicCAS(counters + 1, 0u,
                          (uint32_t)(T.steps > v.nnodes + 1 ? DEV_STEP_CAP : DEV_STACK_OVERFLOW));
            counts[i] = make_uint2(T.cur == kNoRoot ? 0u : T.steps, T.tested);
        });
}

__global__ void __launch_bounds__(kBlock) k_trace_exact(SceneView v, const rt_ray *__restrict__ rays,
                                                        rt_hit *__restrict__ hits, uint32_t flags,
                                                        const uint32_t *__restrict__ queue, uint32_t queue_cap,
                                                        uint32_t *__restrict__ counters)
{
    const uint32_t count = min(*(volatile uint32_t *)counters, queue_cap);
    const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const uint32_t entry = queue[q];
        const uint64_t i = entry & ~kQueueBlocker;
        float4 ra, rb;
        load_ray(rays, i, ra, rb);
        if (flags & kTraceUnbounded) ra.w = INFINITY;
        WatertightRay w = make_watertight(ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w);
        const float ix = fdiv(1.0f, rb.x), iy = fdiv(1.0f, rb.y), iz = fdiv(1.0f, rb.z);
        rt_hit cand = hits[i];
        bool reached = !(entry & kQueueBlocker) && cand.prim >= 0;
        if (reached) {
            // walk the winner's ancestors in the reference tree (the root is never box-tested)
            uint32_t j = v.ref_pos[cand.prim];
            const uint32_t n = v.ntri, root = 2 * n - 2;
            while (n > 1) {
                uint32_t p = n + j / 2;
                if (p >= root) break;
                const float2 *bx = v.ref_boxes + 3 * (size_t)p;
                float2 b0 = __ldg(bx), b1v = __ldg(bx + 1), b2v = __ldg(bx + 2);
                if (!ref_box_test(b0.x, b0.y, b1v.x, b1v.y, b2v.x, b2v.y, ra.x, ra.y, ra.z, ix, iy, iz, ra.w)) {
                    reached = false;
                    break;
                }
                j = p;
            }
        }
        float t = cand.t, b1 = cand.b1, b2 = cand.b2;
        int32_t prim = cand.prim;
        if (!reached) {
            bool overflow = false;
            prim = replay_reference(v, w, ix, iy, iz, shadow, t, b1, b2, overflow);
            if (overflow) atomicCAS(counters + 1, 0u, (uint32_t)DEV_STACK_OVERFLOW);
            atomicAdd(counters + 2, 1u);
        }
        if (prim < 0) t = INFINITY;
        intersect_spheres(v, 0u, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w, shadow, t, prim, b1, b2);
        reinterpret_cast<float4 *>(hits)[i] = make_float4(t, __int_as_float(prim), b1, b2);
    }
}

// One thread per ray; BITS: the warp's 32 results go out as one word (rays 32w .. 32w+31).
template <bool BITS>
__global__ void __launch_bounds__(kBlock) k_trace_any(SceneView v, const rt_ray *__restrict__ rays, uint64_t n,
                                                      void *__restrict__ out, uint32_t flags,
                                                      uint32_t *__restrict__ counters)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool occ = false;
    if (i < n) {
        float4 ra, rb;
        load_ray(rays, i, ra, rb);
        const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
        WatertightRay w = make_watertight(ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w);
        Best best{INFINITY, -1, 0u, 0.f, 0.f, INFINITY};
        bool ok = true;
        if (v.ntri > 0) ok = traverse_bvh8(v, w, rb.x, rb.y, rb.z, shadow, true, best);
        if (!ok) atomicCAS(counters + 1, 0u, (uint32_t)DEV_STACK_OVERFLOW);
        occ = best.prim >= 0 && best.t < ra.w;
        if (!occ) {
            float t = ra.w;
            int32_t prim = -1;
            float b1 = 0, b2 = 0;
            intersect_spheres(v, 0u, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w, shadow, t, prim, b1, b2);
            occ = prim >= 0 && t < ra.w;
        }
    }
    if (BITS) {
        // the grid covers whole warps, so every lane of a warp reaches the ballot
        const uint32_t word = __ballot_sync(0xFFFFFFFFu, occ);
        if ((threadIdx.x & 31u) == 0 && i < n) static_cast<uint32_t *>(out)[i >> 5] = word;
    } else if (i < n) {
        static_cast<uint8_t *>(out)[i] = occ ? 1 : 0;
    }
}

// Scene::isVisible's decision from the closest hits of an unbounded trace: a ray is
// occluded when it hit something no farther than its tmax (visible = no hit or t > distance).
template <bool BITS>
__global__ void __launch_bounds__(kBlock) k_occlusion_from_hits(const rt_ray *__restrict__ rays, uint64_t n,
                                                                const rt_hit *__restrict__ hits, void *__restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool occ = false;
    if (i < n) {
        const float4 h = __ldg(reinterpret_cast<const float4 *>(hits) + i);
        const float tmax = __ldg(reinterpret_cast<const float *>(rays) + 8 * i + 3);
        occ = __float_as_int(h.y) != RT_PRIM_NONE && h.x <= tmax;
    }
    if (BITS) {
        const uint32_t word = __ballot_sync(0xFFFFFFFFu, occ);
        if ((threadIdx.x & 31u) == 0 && i < n) static_cast<uint32_t *>(out)[i >> 5] = word;
    } else if (i < n) {
        static_cast<uint8_t *>(out)[i] = occ ? 1 : 0;
    }
}

}  // namespace

// Resident blocks of the persistent closest-hit kernel on the current device.
static unsigned persistent_blocks()
{
    unsigned cached = device_slot(SLOT_TRACE_RESIDENT);
    if (!cached) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_closest, kBlock, 0);
        cached = device_sm_count() * (unsigned)std::max(per_sm, 1);
        set_device_slot(SLOT_TRACE_RESIDENT, cached);
    }
    return cached;
}

// Grid of k_trace_exact: a grid-stride loop over the (usually tiny) replay queue, four
// blocks per SM.
static unsigned exact_blocks() { return 4 * device_sm_count(); }

int launch_trace_closest(const SceneView &v, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags,
                         uint32_t *queue, uint32_t queue_cap, uint32_t *counters, cudaStream_t s)
{
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s));
    const uint64_t blocks = std::min<uint64_t>((n + kBlock - 1) / kBlock, persistent_blocks());
    k_trace_closest<<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, n, nullptr, hits, flags, queue, queue_cap, counters);
    RTB_CUDA(cudaGetLastError());
    // Always launched: stack-overflow rays are replayed even in RT_TRACE_FAST mode. It
    // reads the queue length on the device, so no host synchronisation is needed.
    k_trace_exact<<<exact_blocks(), kBlock, 0, s>>>(v, rays, hits, flags, queue, queue_cap, counters);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

int launch_trace_closest_dev(const SceneView &v, const rt_ray *rays, const uint32_t *n_dev, uint32_t cap, rt_hit *hits,
                             uint32_t flags, uint32_t *queue, uint32_t *counters, cudaStream_t s)
{
    if (cap == 0) return RT_OK;
    RTB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s));
    const uint64_t blocks = std::min<uint64_t>(((uint64_t)cap + kBlock - 1) / kBlock, persistent_blocks());
    k_trace_closest<<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, cap, n_dev, hits, flags, queue, cap, counters);
    RTB_CUDA(cudaGetLastError());
    k_trace_exact<<<exact_blocks(), kBlock, 0, s>>>(v, rays, hits, flags, queue, cap, counters);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

int launch_trace_counts(const SceneView &v, const rt_ray *rays, uint64_t n, uint32_t flags, bool anyhit,
                        uint32_t *counts, uint32_t *counters, cudaStream_t s)
{
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s));
    const uint64_t blocks = std::min<uint64_t>((n + kBlock - 1) / kBlock, persistent_blocks());
    k_trace_counts<<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, n, flags, anyhit, reinterpret_cast<uint2 *>(counts),
                                                       counters);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

int launch_occlusion_from_hits(const rt_ray *rays, uint64_t n, const rt_hit *hits, void *out, bool bits, cudaStream_t s)
{
    if (n == 0) return RT_OK;
    const uint64_t blocks = (n + kBlock - 1) / kBlock;
    if (bits)
        k_occlusion_from_hits<true><<<(unsigned)blocks, kBlock, 0, s>>>(rays, n, hits, out);
    else
        k_occlusion_from_hits<false><<<(unsigned)blocks, kBlock, 0, s>>>(rays, n, hits, out);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

int launch_trace_any(const SceneView &v, const rt_ray *rays, uint64_t n, void *out, bool bits, uint32_t flags,
                     uint32_t *counters, cudaStream_t s)
{
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s));
    const uint64_t blocks = (n + kBlock - 1) / kBlock;
    if (bits)
        k_trace_any<true><<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, n, out, flags, counters);
    else
        k_trace_any<false><<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, n, out, flags, counters);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

}  // namespace rtb
