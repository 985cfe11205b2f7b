// Reference-order tree: the binary BVH the reference builds (BVH::BVH,
// cuda_libraries/BVH.cu:314-341), rebuilt on the host so the GPU traversal can
// (1) break exact distance ties with the reference's static traversal order and
// (2) replay the reference traversal for the rare rays where order matters.
//
// Steps restated (own code, same arithmetic):
//   * scene bound = Bound3f() (the degenerate box at the origin, BoundingBox.cu:16-21)
//     merged with every triangle's bound (Triangle.cu:123-131, 742-746);
//   * centroid = (1/3) * ((p0 + p1) + p2) (Triangle.cu:657-664, Point.cu:147-151);
//   * unit-cube coordinates (BoundingBox.cu:176-183) and the 30-bit Morton code with its
//     clamps evaluated in double (geometricMath.cu:16-44);
//   * ascending sort of (code, triangle id) pairs (Triangle.cu:759-775);
//   * FIFO pairing (BVH.cu:153-201): node i < 2n-2 hangs from node n + i/2, as the left
//     child when i is even; root = 2n-2; interior boxes merged in index order
//     (BVH.cu:203-212).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <thread>

#include "bvh_common.cuh"
#include "rt_internal.h"

namespace rtb {
namespace {

template <typename F>
void parallel_chunks(uint32_t n, F &&f)
{
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 65536) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) {
        uint32_t b = (uint32_t)((uint64_t)n * t / nt), e = (uint32_t)((uint64_t)n * (t + 1) / nt);
        if (nt == 1) {
            f(b, e);
        } else {
            th.emplace_back([=, &f]() { f(b, e); });
        }
    }
    for (auto &x : th) x.join();
}

}  // namespace

void build_ref_tree(const float *tri9, uint32_t n, RefTreeHost &out)
{
    out.codes.assign(n, 0);
    out.sorted.assign(n, 0);
    out.pos.assign(n, 0);
    out.rank.assign(n, 0);
    out.boxes.clear();
    if (n == 0) return;
    out.boxes.assign(6 * (2 * (size_t)n - 1), 0.f);
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (uint64_t i = 0; i < 9 * (uint64_t)n; i++) {
        int c = (int)(i % 3);
        lo[c] = fminf(lo[c], tri9[i]);
        hi[c] = fmaxf(hi[c], tri9[i]);
    }
    const float diag[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    std::vector<uint64_t> keys(n);
    parallel_chunks(n, [&](uint32_t b, uint32_t e) {
        for (uint32_t t = b; t < e; t++) keys[t] = ref_sort_key(tri9 + 9 * (size_t)t, t, lo, diag);
    });
    std::sort(keys.begin(), keys.end());
    for (uint32_t i = 0; i < n; i++) {
        out.codes[i] = (uint32_t)(keys[i] >> 32);
        out.sorted[i] = (uint32_t)keys[i];
        out.pos[out.sorted[i]] = i;
    }
    float *bx = out.boxes.data();
    for (uint32_t i = 0; i < n; i++) {
        const float *p = tri9 + 9 * (size_t)out.sorted[i];
        for (int c = 0; c < 3; c++) {
            float mn = fminf(p[c], p[3 + c]), mx = fmaxf(p[c], p[3 + c]);
            bx[6 * (size_t)i + c] = fminf(mn, p[6 + c]);
            bx[6 * (size_t)i + 3 + c] = fmaxf(mx, p[6 + c]);
        }
    }
    for (size_t i = n; i + 1 < 2 * (size_t)n; i++) {
        size_t l = 2 * (i - n), r = l + 1;
        for (int c = 0; c < 3; c++) {
            bx[6 * i + c] = fminf(bx[6 * l + c], bx[6 * r + c]);
            bx[6 * i + 3 + c] = fmaxf(bx[6 * l + 3 + c], bx[6 * r + 3 + c]);
        }
    }
    // Static traversal order of BVH::intersectRay (BVH.cu:392-445): at each pop the leaf
    // children are tested left then right; interior children are pushed left then right,
    // so the right subtree is visited before the left one.
    if (n == 1) {
        out.rank[out.sorted[0]] = 0;
        return;
    }
    std::vector<uint32_t> stack;
    stack.reserve(128);
    stack.push_back(2 * n - 2);
    uint32_t next = 0;
    while (!stack.empty()) {
        uint32_t node = stack.back();
        stack.pop_back();
        uint32_t ch[2] = {2 * (node - n), 2 * (node - n) + 1};
        for (int k = 0; k < 2; k++) {
            if (ch[k] < n)
                out.rank[out.sorted[ch[k]]] = next++;
            else
                stack.push_back(ch[k]);
        }
    }
}

}  // namespace rtb
