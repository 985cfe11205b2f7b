// Host builder of the compressed 8-wide BVH traversed by the sm_100a kernels (the device
// builder, build_gpu.cu, produces the same bytes):
//
//   1. binary BVH by PLOC over the Morton order of the reference-order tree: clusters merge
//      with their mutual nearest neighbour (smallest union area within kPlocRadius) until
//      one is left (Meister and Bittner, "Parallel Locally-Ordered Clustering for Bounding
//      Volume Hierarchy Construction", IEEE TVCG 2018);
//   2. triangles numbered in depth-first order (left child first), so every subtree is one
//      range, and subtrees of at most 3 triangles turned into leaves by the SAH rule;
//   3. collapse to 8-wide nodes, breadth first, by repeatedly opening the interior child with
//      the largest surface area; each node's interior children are contiguous, and so are
//      the triangle records of its leaves;
//   4. child boxes quantized to 8 bits per axis on a power-of-two grid, rounded outward and
//      checked in float so that every dequantized box contains the child's box enlarged by
//      the scene margin.
#include <algorithm>
#include <cstring>
#include <deque>

#include "bvh_common.cuh"
#include "rt_internal.h"

namespace rtb {

void build_bvh8(const float *tri9, uint32_t n, float margin, const uint32_t *sorted, uint32_t radius,
                Bvh8Host &out)
{
    out.nodes.clear();
    out.leaf_tris.clear();
    if (n == 0) return;
    // binary nodes: internal 0..n-2 in creation order (root n-2), leaf p (Morton position) n - 1 + p
    const size_t nb = 2 * (size_t)n - 1;
    std::vector<BBox> box(nb);
    std::vector<uint32_t> c0(n), c1(n);
    for (uint32_t p = 0; p < n; p++) box[n - 1 + p] = triangle_box(tri9 + 9 * (size_t)sorted[p], margin);
    // 1. PLOC
    std::vector<uint32_t> cl(n), nn(n), next;
    for (uint32_t p = 0; p < n; p++) cl[p] = n - 1 + p;
    uint32_t made = 0;
    while (cl.size() > 1) {
        const int64_t m = (int64_t)cl.size();
        for (int64_t i = 0; i < m; i++)
            nn[i] = (uint32_t)ploc_nearest(i, m, radius, [&](int64_t j) { return box[cl[j]]; });
        next.clear();
        for (int64_t i = 0; i < m; i++) {
            const uint32_t j = nn[i];
            if (nn[j] == (uint32_t)i) {
                if ((uint32_t)i < j) {  // the lower index of a mutual pair makes the node
                    const uint32_t k = made++;
                    c0[k] = cl[i];
                    c1[k] = cl[j];
                    box[k] = box[cl[i]];
                    bbox_grow(box[k], box[cl[j]]);
                    next.push_back(k);
                }
            } else {
                next.push_back(cl[i]);
            }
        }
        cl.swap(next);
    }
    const uint32_t root = cl[0];
    // 2. depth-first numbering and leaves
    std::vector<uint32_t> size(nb, 1), first(nb, 0), ids(n);
    for (uint32_t k = 0; k + 1 < n; k++) size[k] = size[c0[k]] + size[c1[k]];  // children made first
    for (int64_t k = (int64_t)n - 2; k >= 0; k--) {  // parents made after their children
        first[c0[k]] = first[k];
        first[c1[k]] = first[k] + size[c0[k]];
    }
    for (uint32_t p = 0; p < n; p++) ids[first[n - 1 + p]] = sorted[p];
    std::vector<uint8_t> leaf(nb, 1);
    for (uint32_t k = 0; k + 1 < n; k++)
        leaf[k] = sah_leaf(size[k], bbox_area(box[k]), bbox_area(box[c0[k]]), size[c0[k]], bbox_area(box[c1[k]]),
                           size[c1[k]]);
    auto is_leaf = [&](uint32_t x) { return leaf[x] != 0; };
    auto child = [&](uint32_t x, int s) { return s ? c1[x] : c0[x]; };
    auto area = [&](uint32_t x) { return bbox_area(box[x]); };
    auto box_of = [&](uint32_t x) { return box[x]; };
    auto leaf_range = [&](uint32_t x, uint32_t &f, uint32_t &c) {
        f = first[x];
        c = size[x];
    };
    // 3-4. collapse, breadth first
    out.nodes.reserve(n / 2 + 8);
    out.leaf_tris.resize(n);
    std::deque<std::pair<uint32_t, uint32_t>> q;  // binary node, wide node
    out.nodes.emplace_back();
    q.push_back({root, 0});
    uint32_t ntris = 0;
    while (!q.empty()) {
        const auto it = q.front();
        q.pop_front();
        uint32_t ch[8];
        const int nch = wide_children(it.first, ch, is_leaf, child, area);
        const uint32_t base = (uint32_t)out.nodes.size();
        Bvh8Node node;
        uint32_t toff = 0;
        write_wide_node(
            node, ch, nch, base, ntris, is_leaf, leaf_range, box_of,
            [&](uint32_t rec, uint32_t pos) {
                out.leaf_tris[rec] = ids[pos];
                toff++;
            },
            [&](uint32_t k, uint32_t x) {
                out.nodes.emplace_back();
                q.push_back({x, base + k});
            });
        ntris += toff;
        out.nodes[it.second] = node;
    }
}

}  // namespace rtb
