// BVH8 traversal and reference replay shared by the trace and render kernels.
// See trace.cu for the parity argument.
#pragma once

#include <cfloat>

#include "exact_math.cuh"
#include "rt_internal.h"

namespace rtb {

// Entries of a walk's stack (8 bytes each, in local memory). A walk that would need more ends,
// and its ray is replayed on the reference tree (exact); 32 entries overflowed on dense
// triangle soups without changing the render's speed.
#ifndef RTB_KSTACK
#define RTB_KSTACK 48
#endif
constexpr int kStack = RTB_KSTACK;

// Resident blocks of 128 threads per SM the traversal kernels are compiled for (register cap
// 65536 / (128 * N)): 9 gives 56 registers and 36 warps per SM (measured on the BVH-stress
// ray set: 2294 / 2410 / 2490 Mrays/s for 7 / 8 / 9 with the binned-SAH tree; 3134 / 2870 /
// 2530 for 9 / 10 (48 registers) / 11 (40) with the PLOC tree).
#ifndef RTB_TRAV_MIN_BLOCKS
#define RTB_TRAV_MIN_BLOCKS 9
#endif
constexpr uint32_t kQueueBlocker = 0x80000000u;  // queue entry flag: replay needed (not just ancestor walk)

struct Best {
    float t;
    int32_t prim;
    uint32_t rank;
    float b1, b2;
    float minblock;
};

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int k) { return (w >> (8 * k)) & 0xFFu; }

// Scene records (nodes, triangles) and streamed rays. Evict-last L2 policies on the scene loads
// with evict-first ray loads were measured against these plain read-only loads: 3207 against 3183
// Mrays/s on the 2^24 BVH-stress rays, 1821 against 1832 on the render; not kept.
__device__ __forceinline__ uint4 ld_scene(const uint4 *ptr) { return __ldg(ptr); }
__device__ __forceinline__ float4 ld_scene(const float4 *ptr) { return __ldg(ptr); }
__device__ __forceinline__ float4 ld_stream(const float4 *ptr) { return __ldg(ptr); }

__device__ __forceinline__ void load_ray(const rt_ray *rays, uint64_t i, float4 &a, float4 &b)
{
    const float4 *r4 = reinterpret_cast<const float4 *>(rays);
    a = ld_stream(r4 + 2 * i);
    b = ld_stream(r4 + 2 * i + 1);
}

// Tests one triangle record against the running best; see the file comment for the rule.
__device__ __forceinline__ void test_triangle(const WatertightRay &w, const TriRecord *tris, uint32_t rec,
                                              bool shadow, Best &best)
{
    const float4 *p = reinterpret_cast<const float4 *>(tris + rec);
    float4 a = ld_scene(p), b = ld_scene(p + 1), c = ld_scene(p + 2);
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

// Per-ray traversal state of the BVH8 walk. The walk advances one node per trav_step so a
// persistent warp can retire finished rays and start new ones lane by lane.
struct Trav {
    WatertightRay w;
    float dx, dy, dz;
    float ix, iy, iz, oix, oiy, oiz;
    uint32_t cur;
    int sp;
    uint32_t steps;
    bool ok;
    bool shadow;  // checkShadow semantics: transparent primitives are skipped
    Best best;
    uint32_t tested;  // triangle records tested (counted by the COUNT walk only; steps counts nodes)
    // node index, entry distance bits: one 8-byte local access per push / pop. Keeping the bottom
    // 4 or 8 entries in shared memory instead (the rest in local memory) measured slower, render
    // 2091 / 2100 against 2210 Mrays/s and 2^24-ray trace ~2800 against ~3100: the choice
    // between the two memories at every push and pop costs registers (spills from 32 to 344
    // bytes) and instructions that the saved local traffic does not repay
    uint2 st[kStack];
};

// BVH8 root of scene `sub` (0 for a plain scene) and its spheres [s0, s0 + ns).
__device__ __forceinline__ uint32_t scene_root(const SceneView &v, uint32_t sub)
{
    if (v.subs) return v.subs[min(sub, v.nsubs - 1)].root;
    return v.ntri ? 0u : kNoRoot;
}
__device__ __forceinline__ void scene_spheres(const SceneView &v, uint32_t sub, uint32_t &s0, uint32_t &ns)
{
    if (v.subs) {
        const SubScene &ss = v.subs[min(sub, v.nsubs - 1)];
        s0 = ss.sph0;
        ns = ss.nsph;
    } else {
        s0 = 0;
        ns = v.nspheres;
    }
}

// root: the BVH8 node the walk starts at (kNoRoot: the scene has no triangles; the walk is
// skipped).
__device__ __forceinline__ void trav_init(Trav &T, float ox, float oy, float oz, float dx, float dy, float dz,
                                          float tmax, uint32_t root)
{
    T.w = make_watertight(ox, oy, oz, dx, dy, dz, tmax);
    T.dx = dx;
    T.dy = dy;
    T.dz = dz;
    T.ix = 1.0f / dx;
    T.iy = 1.0f / dy;
    T.iz = 1.0f / dz;
    T.oix = -ox * T.ix;
    T.oiy = -oy * T.iy;
    T.oiz = -oz * T.iz;
    T.cur = root;
    T.sp = 0;
    T.steps = 0;
    T.ok = true;
    T.shadow = false;
    T.best = Best{INFINITY, -1, 0u, 0.f, 0.f, INFINITY};
    T.tested = 0;
}

// Visits node T.cur: tests its eight quantized child boxes (unrolled), the triangles of the
// hit leaves (rolled, so the long exact triangle test exists once in the instruction
// stream), pushes the hit interior children far-to-near and selects the next node.
// Postponing the leaf tests to separate warp-wide triangle steps (one triangle per lane per
// step, taken when enough lanes have triangles waiting) visits the same nodes in the same
// order but was slower on the BVH-stress scene: render 1683 / 1714 / 1654 against 1832
// Mrays/s, 2^24-ray trace ~2900 against 3123, for triangle-step ratios 3 / 2 / 5 (leaves
// hold at most 3 triangles, so the per-step phase vote costs more than the packing saves).
// Two smaller rewrites of the box test were slower too (render / trace Mrays/s, against
// 1837 / 3130): bytes turned into floats through the mantissa of 2^23 (1815 / 3067), and a
// minimum instead of the sorting network when one interior child is hit (1824 / 3086). Shadow
// rays (any hit) gain from the near-to-far order too: pushing their children unsorted, or only
// the nearest first, rendered at 2140 and 2112 against 2228 Mrays/s (2^26 paths).
// Returns true when the ray is done (T.ok = false if the stack or step cap was exceeded).
template <bool COUNT = false>
__device__ __forceinline__ bool trav_step(const SceneView &v, Trav &T, bool anyhit)
{
    const bool shadow = T.shadow;
    if (++T.steps > v.nnodes + 1) {
        T.ok = false;
        return true;
    }
    const uint4 *np = reinterpret_cast<const uint4 *>(v.nodes + T.cur);
    const uint4 n0 = ld_scene(np), n1 = ld_scene(np + 1), n2 = ld_scene(np + 2), n3 = ld_scene(np + 3),
                n4 = ld_scene(np + 4);
    const float sx = __uint_as_float((n0.w & 0xFFu) << 23);
    const float sy = __uint_as_float(((n0.w >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((n0.w >> 16) & 0xFFu) << 23);
    const uint32_t imask = n0.w >> 24;
    const uint32_t child_base = n1.x, tri_base = n1.y;
    const uint32_t meta_lo = n1.z, meta_hi = n1.w;
    // per-axis affine map t = q * (s * inv) + (p * inv - o * inv)
    const float ax = sx * T.ix, bx = fmaf(__uint_as_float(n0.x), T.ix, T.oix);
    const float ay = sy * T.iy, by = fmaf(__uint_as_float(n0.y), T.iy, T.oiy);
    const float az = sz * T.iz, bz = fmaf(__uint_as_float(n0.z), T.iz, T.oiz);
    const float tlimit = fminf(T.best.t, T.w.tmax);
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
#pragma unroll 1
    while (leafmask) {
        const int k = __ffs(leafmask) - 1;
        leafmask &= leafmask - 1;
        const uint32_t meta = byte_of(k < 4 ? meta_lo : meta_hi, k & 3);
        const uint32_t first = tri_base + (meta & 31u), cnt = (meta >> 5) + 1;
        if (COUNT) T.tested += cnt;
#pragma unroll 1
        for (uint32_t j = 0; j < cnt; j++) test_triangle(T.w, v.tris, first + j, shadow, T.best);
        if (anyhit && T.best.prim >= 0) return true;
    }
    uint32_t next = 0xFFFFFFFFu;
    const float tl = fminf(T.best.t, T.w.tmax);
    if (nint) {
        sort8(keys);
#pragma unroll
        for (int j = 7; j >= 1; j--) {
            if (j < (int)nint) {
                const uint32_t slot = keys[j] & 7u;
                const float tn = __uint_as_float(keys[j] & ~7u);
                if (tn <= tl) {
                    if (T.sp >= kStack) {
                        T.ok = false;
                        return true;
                    }
                    T.st[T.sp] = make_uint2(child_base + byte_of(slot < 4 ? meta_lo : meta_hi, slot & 3),
                                            __float_as_uint(tn));
                    T.sp++;
                }
            }
        }
        const uint32_t slot = keys[0] & 7u;
        if (__uint_as_float(keys[0] & ~7u) <= tl) next = child_base + byte_of(slot < 4 ? meta_lo : meta_hi, slot & 3);
    }
    if (next == 0xFFFFFFFFu) {
#pragma unroll 1
        while (T.sp > 0) {
            T.sp--;
            const uint2 e = T.st[T.sp];
            if (__uint_as_float(e.y) <= tl) {
                next = e.x;
                break;
            }
        }
    }
    if (next == 0xFFFFFFFFu) return true;
    T.cur = next;
    return false;
}

// Whole traversal of one ray; returns false if the stack would overflow (result then
// unreliable).
__device__ __forceinline__ bool traverse_bvh8(const SceneView &v, const WatertightRay &w, float dx, float dy, float dz,
                                              bool shadow, bool anyhit, Best &best)
{
    Trav T;
    trav_init(T, w.ox, w.oy, w.oz, dx, dy, dz, w.tmax, scene_root(v, 0));
    T.shadow = shadow;
    T.best = best;
    if (T.cur != kNoRoot)
        while (!trav_step(v, T, anyhit)) {
        }
    best = T.best;
    return T.ok;
}

// Persistent-warp driver: every lane runs its own ray; a lane whose ray is done fetches the
// next ray index from *work (one atomic per fetching warp) until n is exhausted.
// init(i, T) prepares ray i (trav_init + T.shadow), finish(i, T) consumes the result.
// COUNT: the walk also counts the triangle records it tests (T.tested), for rt_trace_counts.
template <bool COUNT = false, typename Init, typename Finish>
__device__ __forceinline__ void persistent_traverse(const SceneView &v, uint32_t n, uint32_t *work, bool anyhit,
                                                    Init init, Finish finish)
{
    const unsigned lane = threadIdx.x & 31u;
    uint32_t ray = 0xFFFFFFFFu;
    bool exhausted = false;
    Trav T;
    for (;;) {
        const bool idle = ray == 0xFFFFFFFFu;
        const unsigned idle_mask = __ballot_sync(0xFFFFFFFFu, idle);
        if (idle_mask && !exhausted) {
            const unsigned leader = __ffs(idle_mask) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(work, (uint32_t)__popc(idle_mask));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (base >= n) exhausted = true;
            if (idle) {
                const uint32_t mine = base + __popc(idle_mask & ((1u << lane) - 1u));
                if (mine < n) {
                    ray = mine;
                    init(ray, T);
                }
            }
        }
        if (__all_sync(0xFFFFFFFFu, ray == 0xFFFFFFFFu)) break;
        if (ray != 0xFFFFFFFFu) {
            if (T.cur == kNoRoot || trav_step<COUNT>(v, T, anyhit)) {
                finish(ray, T);
                ray = 0xFFFFFFFFu;
            }
        }
    }
}

// Scene::intersects' loop over the analytic shapes (Scene.cu:141-146) of scene `sub`.
__device__ __forceinline__ void intersect_spheres(const SceneView &v, uint32_t sub, float ox, float oy, float oz,
                                                  float dx, float dy, float dz, float tmax, bool shadow, float &t,
                                                  int32_t &prim, float &b1, float &b2)
{
    uint32_t s0, ns;
    scene_spheres(v, sub, s0, ns);
    for (uint32_t s = s0; s < s0 + ns; s++) {
        const SphereRecord &sr = v.spheres[s];
        if (shadow && (sr.flags & 1u)) continue;
        float ts, pu = 0.f, pv = 0.f;
        const bool hit = (sr.flags & kShapePlane) ? plane_test(sr.w2o, ox, oy, oz, dx, dy, dz, tmax, ts, pu, pv)
                                                  : sphere_test(sr.w2o, sr.radius, ox, oy, oz, dx, dy, dz, tmax, ts);
        if (hit && ts < t) {
            t = ts;
            prim = RT_PRIM_SHAPE | (int32_t)s;
            b1 = pu;  // a plane hit reports its object-space (x, y); 0 for spheres
            b2 = pv;
        }
    }
}

// Replays BVH::intersectRay on the reference tree for one ray (BVH.cu:355-448).
__device__ __noinline__ static int32_t replay_reference(const SceneView &v, const WatertightRay &w, float ix, float iy, float iz,
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


}  // namespace rtb
