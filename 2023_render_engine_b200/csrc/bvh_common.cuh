// Arithmetic shared by the host and the device builders of the acceleration structures: the
// same floating-point operations in the same order on both sides (the device through the
// round-to-nearest intrinsics, the host without contraction), so that the device build
// reproduces the host build bit for bit.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#include "rt_internal.h"

namespace rtb {

__host__ __device__ __forceinline__ float bv_add(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ float bv_sub(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ float bv_mul(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ float bv_div(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
// std::min / std::max semantics (the first argument unless the second is strictly beyond it)
__host__ __device__ __forceinline__ float bv_min(float a, float b) { return b < a ? b : a; }
__host__ __device__ __forceinline__ float bv_max(float a, float b) { return a < b ? b : a; }

struct BBox {
    float lo[3], hi[3];
};

__host__ __device__ __forceinline__ BBox bbox_empty()
{
    BBox b;
    for (int c = 0; c < 3; c++) {
        b.lo[c] = FLT_MAX;
        b.hi[c] = -FLT_MAX;
    }
    return b;
}

__host__ __device__ __forceinline__ void bbox_grow(BBox &a, const BBox &b)
{
    for (int c = 0; c < 3; c++) {
        a.lo[c] = bv_min(a.lo[c], b.lo[c]);
        a.hi[c] = bv_max(a.hi[c], b.hi[c]);
    }
}

__host__ __device__ __forceinline__ void bbox_grow(BBox &a, const float *p)
{
    for (int c = 0; c < 3; c++) {
        a.lo[c] = bv_min(a.lo[c], p[c]);
        a.hi[c] = bv_max(a.hi[c], p[c]);
    }
}

__host__ __device__ __forceinline__ float bbox_area(const BBox &b)
{
    float d[3];
    for (int c = 0; c < 3; c++) d[c] = bv_max(0.f, bv_sub(b.hi[c], b.lo[c]));
    return bv_mul(2.f, bv_add(bv_add(bv_mul(d[0], d[1]), bv_mul(d[1], d[2])), bv_mul(d[2], d[0])));
}

// Surface area of the union of two boxes.
__host__ __device__ __forceinline__ float union_area(const BBox &a, const BBox &b)
{
    BBox u = a;
    bbox_grow(u, b);
    return bbox_area(u);
}

// The triangle's box enlarged by `margin` (the conservative leaf box of the 8-wide BVH).
__host__ __device__ __forceinline__ BBox triangle_box(const float *p, float margin)
{
    BBox b = bbox_empty();
    for (int k = 0; k < 3; k++) bbox_grow(b, p + 3 * k);
    for (int c = 0; c < 3; c++) {
        b.lo[c] = bv_sub(b.lo[c], margin);
        b.hi[c] = bv_add(b.hi[c], margin);
    }
    return b;
}

// SAH rule that turns a subtree of `cnt` triangles (children of nl and nr) into one leaf: a
// leaf when cnt <= kMaxLeaf and cnt is not above the cost of keeping the split
// (traversal cost 1, intersection cost 1 per triangle). 2^24-ray trace on the BVH-stress scene,
// Mrays/s (BVH8 nodes): 3133 (268,797) for this rule; 3143 (274,795) with leaves of at most 2,
// 3122 (267,843) at most 4; traversal cost 1.5: ~3016 (191,677), 2: 2994 (183,921), 2 with
// leaves of at most 4: 2885 (151,352).
constexpr uint32_t kMaxLeaf = 3;
__host__ __device__ __forceinline__ bool sah_leaf(uint32_t cnt, float parea, float al, uint32_t nl, float ar, uint32_t nr)
{
    if (cnt > kMaxLeaf) return false;
    const float split_cost =
        bv_add(1.0f, parea > 0 ? bv_div(bv_add(bv_mul(al, (float)nl), bv_mul(ar, (float)nr)), parea) : (float)cnt);
    return (float)cnt <= split_cost;
}

// Morton code of the reference (geometricMath.cu:16-44): 10 bits per axis of the unit-cube
// coordinate, the clamps evaluated in double.
__host__ __device__ __forceinline__ uint32_t expand_bits10(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__host__ __device__ __forceinline__ uint32_t ref_morton3d(float x, float y, float z)
{
    x = (float)fmin(fmax((double)x * 1024.0, 0.0), 1023.0);
    y = (float)fmin(fmax((double)y * 1024.0, 0.0), 1023.0);
    z = (float)fmin(fmax((double)z * 1024.0, 0.0), 1023.0);
    return expand_bits10((uint32_t)x) * 4 + expand_bits10((uint32_t)y) * 2 + expand_bits10((uint32_t)z);
}

// Sort key of triangle t for the reference-order tree: its Morton code over the scene box
// (lo, diag) of the centroid (1/3) * ((p0 + p1) + p2) (Triangle.cu:657-664,
// BoundingBox.cu:176-183), then the triangle id.
__host__ __device__ __forceinline__ uint64_t ref_sort_key(const float *p, uint32_t t, const float lo[3],
                                                          const float diag[3])
{
    const float third = (float)1 / 3.0f;
    float u[3];
    for (int c = 0; c < 3; c++) {
        const float cen = bv_mul(third, bv_add(bv_add(p[c], p[3 + c]), p[6 + c]));
        u[c] = bv_div(bv_sub(cen, lo[c]), diag[c]);
    }
    return ((uint64_t)ref_morton3d(u[0], u[1], u[2]) << 32) | t;
}

__host__ __device__ __forceinline__ float bv_frexp_exp(float x, int *e)
{
#ifdef __CUDA_ARCH__
    return frexpf(x, e);
#else
    return std::frexp(x, e);
#endif
}
__host__ __device__ __forceinline__ float bv_ldexp(float x, int e)
{
#ifdef __CUDA_ARCH__
    return ldexpf(x, e);
#else
    return std::ldexp(x, e);
#endif
}
__host__ __device__ __forceinline__ float bv_floor(float x)
{
#ifdef __CUDA_ARCH__
    return floorf(x);
#else
    return std::floor(x);
#endif
}
__host__ __device__ __forceinline__ float bv_ceil(float x)
{
#ifdef __CUDA_ARCH__
    return ceilf(x);
#else
    return std::ceil(x);
#endif
}

// Quantizes the nchild child boxes of an 8-wide node onto a power-of-two grid per axis with
// 8-bit coordinates, rounded outward and checked in float so that every dequantized box
// (p + q * 2^e, the product exact) contains the child box. Sets px..pz, ex..ez and q*.
__host__ __device__ inline void quantize_node(Bvh8Node &out, const BBox *cbox, int nchild)
{
    BBox nb = bbox_empty();
    for (int i = 0; i < nchild; i++) bbox_grow(nb, cbox[i]);
    out.px = nb.lo[0];
    out.py = nb.lo[1];
    out.pz = nb.lo[2];
    float p[3] = {nb.lo[0], nb.lo[1], nb.lo[2]};
    float scale[3];
    uint8_t e8[3];
    for (int a = 0; a < 3; a++) {
        const float ext = bv_sub(nb.hi[a], nb.lo[a]);
        int e = -126;
        if (ext > 0) {
            int ex;
            bv_frexp_exp(bv_div(ext, 255.0f), &ex);  // ext/255 = m * 2^ex, m in [0.5, 1)
            e = ex > -126 ? ex : -126;               // 2^ex >= ext/255
            while (bv_ldexp(255.0f, e) < bv_mul(ext, 1 + 1e-6f)) e++;
        }
        e8[a] = (uint8_t)(e + 127);
        scale[a] = bv_ldexp(1.0f, e);
    }
    out.ex = e8[0];
    out.ey = e8[1];
    out.ez = e8[2];
    uint8_t *qlo[3] = {out.qlox, out.qloy, out.qloz};
    uint8_t *qhi[3] = {out.qhix, out.qhiy, out.qhiz};
    for (int i = 0; i < 8; i++)
        for (int a = 0; a < 3; a++) {
            qlo[a][i] = 0;
            qhi[a][i] = 0;
        }
    for (int i = 0; i < nchild; i++) {
        for (int a = 0; a < 3; a++) {
            const float lo = cbox[i].lo[a], hi = cbox[i].hi[a];
            int ql = (int)bv_floor(bv_div(bv_sub(lo, p[a]), scale[a]));
            int qh = (int)bv_ceil(bv_div(bv_sub(hi, p[a]), scale[a]));
            ql = ql < 0 ? 0 : (ql > 255 ? 255 : ql);
            qh = qh < 0 ? 0 : (qh > 255 ? 255 : qh);
            // the kernel dequantizes as p + q * scale (q * scale is exact): check that in float
            while (ql > 0 && bv_add(p[a], bv_mul((float)ql, scale[a])) > lo) ql--;
            while (qh < 255 && bv_add(p[a], bv_mul((float)qh, scale[a])) < hi) qh++;
            qlo[a][i] = (uint8_t)ql;
            qhi[a][i] = (uint8_t)qh;
        }
    }
}

// PLOC's nearest neighbour of cluster i among clusters [i - radius, i + radius] of m: the
// smallest union area, ties to the lower index.
template <class BoxOf>
__host__ __device__ __forceinline__ int64_t ploc_nearest(int64_t i, int64_t m, uint32_t radius, BoxOf &&box_of)
{
    const BBox a = box_of(i);
    float best = FLT_MAX;
    int64_t bj = -1;
    const int64_t j0 = i > (int64_t)radius ? i - (int64_t)radius : 0;
    const int64_t j1 = i + (int64_t)radius < m - 1 ? i + (int64_t)radius : m - 1;
    for (int64_t j = j0; j <= j1; j++) {
        if (j == i) continue;
        const float s = union_area(a, box_of(j));
        if (s < best) {
            best = s;
            bj = j;
        }
    }
    return bj;
}

// Clusters searched on each side in PLOC. Trace throughput on the 1.31M-triangle BVH-stress
// scene (2^24 rays): radius 8 3132, 16 3018, 24 3019 Mrays/s; binned SAH 2527, Karras LBVH 1652.
constexpr uint32_t kPlocRadius = 8;

// Children of the 8-wide node made from binary node x: its two children, then repeatedly the
// interior child of largest surface area (the first on ties) replaced by its own two, up to 8.
// A leaf x is its own single child (a scene of one leaf). Returns the count.
template <class IsLeaf, class Child, class Area>
__host__ __device__ __forceinline__ int wide_children(uint32_t x, uint32_t ch[8], IsLeaf &&is_leaf, Child &&child,
                                                      Area &&area)
{
    if (is_leaf(x)) {
        ch[0] = x;
        return 1;
    }
    int nch = 2;
    ch[0] = child(x, 0);
    ch[1] = child(x, 1);
    while (nch < 8) {
        int best = -1;
        float ba = -1;
        for (int i = 0; i < nch; i++) {
            if (is_leaf(ch[i])) continue;
            const float a = area(ch[i]);
            if (a > ba) {
                ba = a;
                best = i;
            }
        }
        if (best < 0) break;
        const uint32_t y = ch[best];
        ch[best] = child(y, 0);
        ch[nch++] = child(y, 1);
    }
    return nch;
}

// Fills the 8-wide node for children ch[0..nch): leaf slots hold (count - 1) << 5 | offset into
// the node's block of triangle records (written through leaf_tri(record, triangle)), interior
// slots their rank among the interior children (announced through interior(rank, binary node)).
template <class IsLeaf, class LeafRange, class BoxOf, class LeafTri, class Interior>
__host__ __device__ __forceinline__ void write_wide_node(Bvh8Node &node, const uint32_t ch[8], int nch,
                                                         uint32_t child_base, uint32_t tri_base, IsLeaf &&is_leaf,
                                                         LeafRange &&leaf_range, BoxOf &&box_of, LeafTri &&leaf_tri,
                                                         Interior &&interior)
{
    uint8_t *raw = reinterpret_cast<uint8_t *>(&node);
    for (unsigned i = 0; i < sizeof(Bvh8Node); i++) raw[i] = 0;
    for (int i = 0; i < 8; i++) node.meta[i] = 0xFF;
    node.child_base = child_base;
    node.tri_base = tri_base;
    BBox cbox[8];
    uint32_t ninterior = 0, toff = 0;
    for (int i = 0; i < nch; i++) {
        cbox[i] = box_of(ch[i]);
        if (is_leaf(ch[i])) {
            uint32_t first, count;
            leaf_range(ch[i], first, count);
            node.meta[i] = (uint8_t)(((count - 1) << 5) | toff);
            for (uint32_t k = 0; k < count; k++) leaf_tri(tri_base + toff + k, first + k);
            toff += count;
        } else {
            node.meta[i] = (uint8_t)ninterior;
            node.imask |= (uint8_t)(1u << i);
            interior(ninterior, ch[i]);
            ninterior++;
        }
    }
    quantize_node(node, cbox, nch);
}

}  // namespace rtb
