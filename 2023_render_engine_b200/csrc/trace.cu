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
#include <cfloat>

#include "exact_math.cuh"
#include "rt_internal.h"

namespace rtb {

namespace {

constexpr int kStack = 48;
constexpr int kBlock = 128;
constexpr uint32_t kQueueBlocker = 0x80000000u;  // queue entry flag: replay needed (not just ancestor walk)

struct Best {
    float t;
    int32_t prim;
    uint32_t rank;
    float b1, b2;
    float minblock;
};

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int k) { return (w >> (8 * k)) & 0xFFu; }

__device__ __forceinline__ void load_ray(const rt_ray *rays, uint64_t i, float4 &a, float4 &b)
{
    const float4 *r4 = reinterpret_cast<const float4 *>(rays);
    a = __ldg(r4 + 2 * i);
    b = __ldg(r4 + 2 * i + 1);
}

// Tests one triangle record against the running best; see the file comment for the rule.
__device__ __forceinline__ void test_triangle(const WatertightRay &w, const TriRecord *tris, uint32_t rec,
                                              bool shadow, Best &best)
{
    const float4 *p = reinterpret_cast<const float4 *>(tris + rec);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    if (shadow && (__float_as_uint(c.w) & 1u)) return;
    TriHit h;
    if (!watertight_test(w, a, b, c, h)) return;
    uint32_t rank = __float_as_uint(a.w);
    if (h.t > best.t) return;
    if (h.t == best.t && best.prim >= 0 && rank < best.rank) return;
    float dt = watertight_delta_t(h);
    if (h.t <= dt) {
        best.minblock = fminf(best.minblock, h.t);
        return;
    }
    best.t = h.t;
    best.prim = (int32_t)__float_as_uint(b.w);
    best.rank = rank;
    best.b1 = fmul(h.e1, h.invDet);
    best.b2 = fmul(h.e2, h.invDet);
}

// Sorting network for 8 keys (ascending).
__device__ __forceinline__ void cas(uint32_t &a, uint32_t &b)
{
    uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}
__device__ __forceinline__ void sort8(uint32_t k[8])
{
    cas(k[0], k[1]); cas(k[2], k[3]); cas(k[4], k[5]); cas(k[6], k[7]);
    cas(k[0], k[2]); cas(k[1], k[3]); cas(k[4], k[6]); cas(k[5], k[7]);
    cas(k[1], k[2]); cas(k[5], k[6]); cas(k[0], k[4]); cas(k[3], k[7]);
    cas(k[1], k[5]); cas(k[2], k[6]);
    cas(k[1], k[4]); cas(k[3], k[6]);
    cas(k[2], k[4]); cas(k[3], k[5]);
    cas(k[3], k[4]);
}

// Traverses the BVH8; returns false if the stack would overflow (result then unreliable).
// The eight child boxes are tested in an unrolled block; the triangles of the hit leaves
// are then tested in a rolled loop so the (long) exact triangle test exists once in the
// instruction stream.
__device__ __forceinline__ bool traverse_bvh8(const SceneView &v, const WatertightRay &w, float dx, float dy, float dz,
                                              bool shadow, bool anyhit, Best &best)
{
    const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
    const float oix = -w.ox * ix, oiy = -w.oy * iy, oiz = -w.oz * iz;
    uint32_t st_node[kStack];
    float st_t[kStack];
    int sp = 0;
    uint32_t cur = 0;
    uint32_t steps = 0;
    const uint32_t cap = v.nnodes + 1;
#pragma unroll 1
    for (;;) {
        if (++steps > cap) return false;
        const uint4 *np = reinterpret_cast<const uint4 *>(v.nodes + cur);
        const uint4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
        const float sx = __uint_as_float((n0.w & 0xFFu) << 23);
        const float sy = __uint_as_float(((n0.w >> 8) & 0xFFu) << 23);
        const float sz = __uint_as_float(((n0.w >> 16) & 0xFFu) << 23);
        const uint32_t imask = n0.w >> 24;
        const uint32_t child_base = n1.x, tri_base = n1.y;
        const uint32_t meta_lo = n1.z, meta_hi = n1.w;
        // per-axis affine map t = q * (s * inv) + (p * inv - o * inv)
        const float ax = sx * ix, bx = fmaf(__uint_as_float(n0.x), ix, oix);
        const float ay = sy * iy, by = fmaf(__uint_as_float(n0.y), iy, oiy);
        const float az = sz * iz, bz = fmaf(__uint_as_float(n0.z), iz, oiz);
        const float tlimit = fminf(best.t, w.tmax);
        uint32_t keys[8];
        uint32_t nint = 0, leafmask = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int b = k & 3;
            const uint32_t meta = byte_of(k < 4 ? meta_lo : meta_hi, b);
            const float qlx = (float)byte_of(k < 4 ? n2.x : n2.y, b);
            const float qly = (float)byte_of(k < 4 ? n2.z : n2.w, b);
            const float qlz = (float)byte_of(k < 4 ? n3.x : n3.y, b);
            const float qhx = (float)byte_of(k < 4 ? n3.z : n3.w, b);
            const float qhy = (float)byte_of(k < 4 ? n4.x : n4.y, b);
            const float qhz = (float)byte_of(k < 4 ? n4.z : n4.w, b);
            const float t1x = fmaf(qlx, ax, bx), t2x = fmaf(qhx, ax, bx);
            const float t1y = fmaf(qly, ay, by), t2y = fmaf(qhy, ay, by);
            const float t1z = fmaf(qlz, az, bz), t2z = fmaf(qhz, az, bz);
            const float tn = fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fmaxf(fminf(t1z, t2z), 0.0f));
            const float tf = fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fminf(fmaxf(t1z, t2z), tlimit));
            const bool hit = (meta != 0xFFu) && (tn <= tf);
            const bool interior = (imask >> k) & 1u;
            keys[k] = (hit && interior) ? ((__float_as_uint(tn) & ~7u) | (uint32_t)k) : 0xFFFFFFFFu;
            nint += (hit && interior) ? 1u : 0u;
            leafmask |= (hit && !interior) ? (1u << k) : 0u;
        }
        // leaves: one copy of the exact triangle test
#pragma unroll 1
        while (leafmask) {
            const int k = __ffs(leafmask) - 1;
            leafmask &= leafmask - 1;
            const uint32_t meta = byte_of(k < 4 ? meta_lo : meta_hi, k & 3);
            const uint32_t first = tri_base + (meta & 31u), cnt = (meta >> 5) + 1;
#pragma unroll 1
            for (uint32_t j = 0; j < cnt; j++) test_triangle(w, v.tris, first + j, shadow, best);
            if (anyhit && best.prim >= 0) return true;
        }
        uint32_t next = 0xFFFFFFFFu;
        const float tl = fminf(best.t, w.tmax);
        if (nint) {
            sort8(keys);
            // push far to near (register-resident keys: unrolled with a predicate)
#pragma unroll
            for (int j = 7; j >= 1; j--) {
                if (j < (int)nint) {
                    const uint32_t slot = keys[j] & 7u;
                    const float tn = __uint_as_float(keys[j] & ~7u);
                    if (tn <= tl) {
                        if (sp >= kStack) return false;
                        st_node[sp] = child_base + byte_of(slot < 4 ? meta_lo : meta_hi, slot & 3);
                        st_t[sp] = tn;
                        sp++;
                    }
                }
            }
            const uint32_t slot = keys[0] & 7u;
            if (__uint_as_float(keys[0] & ~7u) <= tl) next = child_base + byte_of(slot < 4 ? meta_lo : meta_hi, slot & 3);
        }
        if (next == 0xFFFFFFFFu) {
#pragma unroll 1
            while (sp > 0) {
                sp--;
                if (st_t[sp] <= tl) {
                    next = st_node[sp];
                    break;
                }
            }
        }
        if (next == 0xFFFFFFFFu) return true;
        cur = next;
    }
}

__device__ __forceinline__ void shade_spheres(const SceneView &v, float ox, float oy, float oz, float dx, float dy,
                                              float dz, float tmax, bool shadow, float &t, int32_t &prim, float &b1,
                                              float &b2)
{
    for (uint32_t s = 0; s < v.nspheres; s++) {
        const SphereRecord &sr = v.spheres[s];
        if (shadow && (sr.flags & 1u)) continue;
        float ts;
        if (sphere_test(sr.w2o, sr.radius, ox, oy, oz, dx, dy, dz, tmax, ts) && ts < t) {
            t = ts;
            prim = RT_PRIM_SHAPE | (int32_t)s;
            b1 = 0.f;
            b2 = 0.f;
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_trace_closest(SceneView v, const rt_ray *__restrict__ rays, uint64_t n,
                                                          rt_hit *__restrict__ hits, uint32_t flags,
                                                          uint32_t *__restrict__ queue, uint32_t queue_cap,
                                                          uint32_t *__restrict__ counters)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 ra, rb;
    load_ray(rays, i, ra, rb);
    const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
    WatertightRay w = make_watertight(ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w);
    Best best{INFINITY, -1, 0u, 0.f, 0.f, INFINITY};
    bool ok = true;
    if (v.ntri > 0) ok = traverse_bvh8(v, w, rb.x, rb.y, rb.z, shadow, false, best);
    bool exact_needed = false, replay = false;
    if (!ok) {
        exact_needed = replay = true;
        atomicCAS(counters + 1, 0u, (uint32_t)DEV_STACK_OVERFLOW);
    } else if (!(flags & RT_TRACE_FAST) && best.prim >= 0) {
        if (best.minblock < best.t) {
            exact_needed = replay = true;
        } else if (!(ra.w == INFINITY) || rb.x == 0.f || rb.y == 0.f || rb.z == 0.f) {
            exact_needed = true;  // ancestor walk in k_trace_exact
        } else {
            const float4 *p = reinterpret_cast<const float4 *>(v.tris + v.leafpos[best.prim]);
            float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
            float lx = fminf(fminf(a.x, b.x), c.x), ly = fminf(fminf(a.y, b.y), c.y), lz = fminf(fminf(a.z, b.z), c.z);
            float hx = fmaxf(fmaxf(a.x, b.x), c.x), hy = fmaxf(fmaxf(a.y, b.y), c.y), hz = fmaxf(fmaxf(a.z, b.z), c.z);
            float ix = fdiv(1.0f, rb.x), iy = fdiv(1.0f, rb.y), iz = fdiv(1.0f, rb.z);
            if (!ref_box_test(lx, ly, lz, hx, hy, hz, ra.x, ra.y, ra.z, ix, iy, iz, ra.w)) exact_needed = true;
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
    shade_spheres(v, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w, shadow, t, prim, b1, b2);
    reinterpret_cast<float4 *>(hits)[i] = make_float4(t, __int_as_float(prim), b1, b2);
}

// Replays BVH::intersectRay on the reference tree for one ray (BVH.cu:355-448).
__device__ int32_t replay_reference(const SceneView &v, const WatertightRay &w, float ix, float iy, float iz,
                                    bool shadow, float &tOut, float &b1, float &b2, bool &overflow)
{
    const uint32_t n = v.ntri;
    float h = INFINITY;
    int32_t hit = -1;
    auto tri_seq = [&](uint32_t tri) {
        const float4 *p = reinterpret_cast<const float4 *>(v.tris + v.leafpos[tri]);
        float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
        if (shadow && (__float_as_uint(c.w) & 1u)) return;
        TriHit th;
        if (!watertight_test(w, a, b, c, th)) return;
        if (th.t > h) return;
        h = th.t;
        if (h <= watertight_delta_t(th)) return;
        hit = (int32_t)tri;
        b1 = fmul(th.e1, th.invDet);
        b2 = fmul(th.e2, th.invDet);
    };
    if (n == 1) {
        tri_seq(v.ref_sorted[0]);
        tOut = h;
        return hit;
    }
    uint32_t stack[64];
    int sp = 0;
    stack[sp++] = 2 * n - 2;
    while (sp > 0) {
        uint32_t node = stack[--sp];
        uint32_t ch0 = 2 * (node - n);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            uint32_t c = ch0 + (uint32_t)k;
            if (c < n) {
                tri_seq(v.ref_sorted[c]);
            } else {
                const float2 *bx = v.ref_boxes + 3 * (size_t)c;
                float2 b0 = __ldg(bx), b1v = __ldg(bx + 1), b2v = __ldg(bx + 2);
                if (ref_box_test(b0.x, b0.y, b1v.x, b1v.y, b2v.x, b2v.y, w.ox, w.oy, w.oz, ix, iy, iz, w.tmax)) {
                    if (sp < 64)
                        stack[sp++] = c;
                    else
                        overflow = true;
                }
            }
        }
    }
    tOut = h;
    return hit;
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
        shade_spheres(v, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w, shadow, t, prim, b1, b2);
        reinterpret_cast<float4 *>(hits)[i] = make_float4(t, __int_as_float(prim), b1, b2);
    }
}

__global__ void __launch_bounds__(kBlock) k_trace_any(SceneView v, const rt_ray *__restrict__ rays, uint64_t n,
                                                      uint8_t *__restrict__ occluded, uint32_t flags,
                                                      uint32_t *__restrict__ counters)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 ra, rb;
    load_ray(rays, i, ra, rb);
    const bool shadow = (flags & RT_TRACE_SHADOW) != 0;
    WatertightRay w = make_watertight(ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w);
    Best best{INFINITY, -1, 0u, 0.f, 0.f, INFINITY};
    bool ok = true;
    if (v.ntri > 0) ok = traverse_bvh8(v, w, rb.x, rb.y, rb.z, shadow, true, best);
    if (!ok) atomicCAS(counters + 1, 0u, (uint32_t)DEV_STACK_OVERFLOW);
    bool occ = best.prim >= 0 && best.t < ra.w;
    if (!occ) {
        float t = ra.w;
        int32_t prim = -1;
        float b1 = 0, b2 = 0;
        shade_spheres(v, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, ra.w, shadow, t, prim, b1, b2);
        occ = prim >= 0 && t < ra.w;
    }
    occluded[i] = occ ? 1 : 0;
}

}  // namespace

int launch_trace_closest(const SceneView &v, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags,
                         uint32_t *queue, uint32_t queue_cap, uint32_t *counters, cudaStream_t s)
{
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s));
    const uint64_t blocks = (n + kBlock - 1) / kBlock;
    k_trace_closest<<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, n, hits, flags, queue, queue_cap, counters);
    RTB_CUDA(cudaGetLastError());
    // Always launched: stack-overflow rays are replayed even in RT_TRACE_FAST mode. It
    // reads the queue length on the device, so no host synchronisation is needed.
    k_trace_exact<<<148 * 4, kBlock, 0, s>>>(v, rays, hits, flags, queue, queue_cap, counters);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

int launch_trace_any(const SceneView &v, const rt_ray *rays, uint64_t n, uint8_t *occluded, uint32_t flags,
                     uint32_t *counters, cudaStream_t s)
{
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s));
    const uint64_t blocks = (n + kBlock - 1) / kBlock;
    k_trace_any<<<(unsigned)blocks, kBlock, 0, s>>>(v, rays, n, occluded, flags, counters);
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

}  // namespace rtb
