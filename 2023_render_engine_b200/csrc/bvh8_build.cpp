// Host builder of the compressed 8-wide BVH traversed by the sm_100a kernels.
//
//   1. binary BVH by binned SAH (32 bins per axis, leaves of at most 3 triangles),
//      subtrees built on parallel host threads;
//   2. collapse to 8-wide nodes by repeatedly opening the interior child with the largest
//      surface area;
//   3. breadth-first layout: each node's interior children are contiguous, and so are the
//      triangle records of its leaves;
//   4. child boxes quantized to 8 bits per axis on a power-of-two grid, rounded outward and
//      checked in float so that every dequantized box contains the child's box enlarged by
//      the scene margin.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <thread>

#include "rt_internal.h"

namespace rtb {
namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const Box &b)
    {
        for (int c = 0; c < 3; c++) {
            lo[c] = std::min(lo[c], b.lo[c]);
            hi[c] = std::max(hi[c], b.hi[c]);
        }
    }
    void grow(const float *p)
    {
        for (int c = 0; c < 3; c++) {
            lo[c] = std::min(lo[c], p[c]);
            hi[c] = std::max(hi[c], p[c]);
        }
    }
    float area() const
    {
        float d[3];
        for (int c = 0; c < 3; c++) d[c] = std::max(0.f, hi[c] - lo[c]);
        return 2.f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

struct BNode {
    Box box;
    int32_t child[2] = {-1, -1};  // interior: children; leaf: -1
    uint32_t first = 0, count = 0;
};

constexpr int kBins = 32;
constexpr uint32_t kMaxLeaf = 3;

struct Builder {
    const std::vector<Box> &prim_box;
    const std::vector<float> &cen;  // 3 per prim
    std::vector<uint32_t> &ids;
    std::vector<BNode> &nodes;
    std::atomic<uint32_t> next{0};

    uint32_t alloc() { return next.fetch_add(1); }

    void make_leaf(uint32_t ni, uint32_t b, uint32_t e)
    {
        BNode &n = nodes[ni];
        n.first = b;
        n.count = e - b;
        n.child[0] = n.child[1] = -1;
    }

    void build(uint32_t ni, uint32_t b, uint32_t e, int depth)
    {
        Box nb, cb;
        for (uint32_t i = b; i < e; i++) {
            nb.grow(prim_box[ids[i]]);
            cb.grow(&cen[3 * (size_t)ids[i]]);
        }
        nodes[ni].box = nb;
        uint32_t cnt = e - b;
        if (cnt <= 1) {
            make_leaf(ni, b, e);
            return;
        }
        // binned SAH over all three axes
        float best_cost = FLT_MAX;
        int best_axis = -1, best_split = -1;
        for (int a = 0; a < 3; a++) {
            float ext = cb.hi[a] - cb.lo[a];
            if (!(ext > 0)) continue;
            Box bins[kBins];
            uint32_t bc[kBins] = {0};
            float k = kBins * (1 - 1e-6f) / ext;
            for (uint32_t i = b; i < e; i++) {
                uint32_t id = ids[i];
                int bi = std::min(kBins - 1, (int)((cen[3 * (size_t)id + a] - cb.lo[a]) * k));
                bins[bi].grow(prim_box[id]);
                bc[bi]++;
            }
            float rarea[kBins];
            uint32_t rcnt[kBins];
            Box acc;
            uint32_t c = 0;
            for (int i = kBins - 1; i > 0; i--) {
                acc.grow(bins[i]);
                c += bc[i];
                rarea[i] = acc.area();
                rcnt[i] = c;
            }
            acc = Box();
            c = 0;
            for (int i = 0; i < kBins - 1; i++) {
                acc.grow(bins[i]);
                c += bc[i];
                if (c == 0 || rcnt[i + 1] == 0) continue;
                float cost = acc.area() * c + rarea[i + 1] * rcnt[i + 1];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_split = i + 1;
                }
            }
        }
        float parea = nb.area();
        float split_cost = 1.0f + (parea > 0 ? best_cost / parea : (float)cnt);
        if (cnt <= kMaxLeaf && (best_axis < 0 || (float)cnt <= split_cost)) {
            make_leaf(ni, b, e);
            return;
        }
        uint32_t mid;
        if (best_axis < 0) {
            mid = b + cnt / 2;  // all centroids coincide: split by count
        } else {
            float ext = cb.hi[best_axis] - cb.lo[best_axis];
            float k = kBins * (1 - 1e-6f) / ext;
            auto it = std::partition(ids.begin() + b, ids.begin() + e, [&](uint32_t id) {
                int bi = std::min(kBins - 1, (int)((cen[3 * (size_t)id + best_axis] - cb.lo[best_axis]) * k));
                return bi < best_split;
            });
            mid = (uint32_t)(it - ids.begin());
            if (mid == b || mid == e) mid = b + cnt / 2;
        }
        uint32_t l = alloc(), r = alloc();
        nodes[ni].child[0] = (int32_t)l;
        nodes[ni].child[1] = (int32_t)r;
        nodes[ni].count = 0;
        if (cnt > 200000 && depth < 5) {
            std::thread t([&, l, b, mid, depth]() { build(l, b, mid, depth + 1); });
            build(r, mid, e, depth + 1);
            t.join();
        } else {
            build(l, b, mid, depth + 1);
            build(r, mid, e, depth + 1);
        }
    }
};

bool is_leaf(const BNode &n) { return n.child[0] < 0; }

void quantize(Bvh8Node &out, const Box *cbox, int nchild)
{
    Box nb;
    for (int i = 0; i < nchild; i++) nb.grow(cbox[i]);
    out.px = nb.lo[0];
    out.py = nb.lo[1];
    out.pz = nb.lo[2];
    float p[3] = {nb.lo[0], nb.lo[1], nb.lo[2]};
    uint8_t e8[3];
    float scale[3];
    for (int a = 0; a < 3; a++) {
        float ext = nb.hi[a] - nb.lo[a];
        int e = -126;
        if (ext > 0) {
            int ex;
            std::frexp(ext / 255.0f, &ex);  // ext/255 = m * 2^ex, m in [0.5, 1)
            e = std::max(-126, ex);         // 2^ex >= ext/255
            while (std::ldexp(255.0f, e) < ext * (1 + 1e-6f)) e++;
        }
        e8[a] = (uint8_t)(e + 127);
        scale[a] = std::ldexp(1.0f, e);
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
            float lo = cbox[i].lo[a], hi = cbox[i].hi[a];
            int ql = (int)std::floor((lo - p[a]) / scale[a]);
            int qh = (int)std::ceil((hi - p[a]) / scale[a]);
            ql = std::max(0, std::min(255, ql));
            qh = std::max(0, std::min(255, qh));
            // the kernel dequantizes as p + q * scale (q * scale is exact): check that in float
            while (ql > 0 && p[a] + (float)ql * scale[a] > lo) ql--;
            while (qh < 255 && p[a] + (float)qh * scale[a] < hi) qh++;
            qlo[a][i] = (uint8_t)ql;
            qhi[a][i] = (uint8_t)qh;
        }
    }
}

}  // namespace

void build_bvh8(const float *tri9, uint32_t n, float margin, Bvh8Host &out)
{
    out.nodes.clear();
    out.leaf_tris.clear();
    if (n == 0) return;
    std::vector<Box> pbox(n);
    std::vector<float> cen(3 * (size_t)n);
    for (uint32_t t = 0; t < n; t++) {
        Box b;
        for (int k = 0; k < 3; k++) b.grow(tri9 + 9 * (size_t)t + 3 * k);
        for (int c = 0; c < 3; c++) {
            b.lo[c] -= margin;
            b.hi[c] += margin;
            cen[3 * (size_t)t + c] = 0.5f * (b.lo[c] + b.hi[c]);
        }
        pbox[t] = b;
    }
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; i++) ids[i] = i;
    std::vector<BNode> bn(2 * (size_t)n);
    Builder bld{pbox, cen, ids, bn};
    uint32_t root = bld.alloc();
    bld.build(root, 0, n, 0);

    // Collapse into 8-wide nodes, breadth first.
    struct Item {
        uint32_t bnode;
        uint32_t wide;
    };
    std::deque<Item> q;
    out.nodes.reserve(n / 2 + 8);
    out.leaf_tris.reserve(n);
    out.nodes.emplace_back();
    q.push_back({root, 0});
    while (!q.empty()) {
        Item it = q.front();
        q.pop_front();
        std::vector<uint32_t> ch;
        if (is_leaf(bn[it.bnode])) {
            ch.push_back(it.bnode);  // a scene with one leaf: the root holds it as its only child
        } else {
            ch.push_back((uint32_t)bn[it.bnode].child[0]);
            ch.push_back((uint32_t)bn[it.bnode].child[1]);
            while (ch.size() < 8) {
                int best = -1;
                float ba = -1;
                for (size_t i = 0; i < ch.size(); i++) {
                    if (is_leaf(bn[ch[i]])) continue;
                    float a = bn[ch[i]].box.area();
                    if (a > ba) {
                        ba = a;
                        best = (int)i;
                    }
                }
                if (best < 0) break;
                uint32_t x = ch[best];
                ch[best] = (uint32_t)bn[x].child[0];
                ch.push_back((uint32_t)bn[x].child[1]);
            }
        }
        Bvh8Node node;
        std::memset(&node, 0, sizeof(node));
        std::memset(node.meta, 0xFF, 8);
        node.child_base = (uint32_t)out.nodes.size();
        node.tri_base = (uint32_t)out.leaf_tris.size();
        Box cbox[8];
        int ninterior = 0;
        uint32_t toff = 0;
        for (size_t i = 0; i < ch.size(); i++) {
            const BNode &c = bn[ch[i]];
            cbox[i] = c.box;
            if (is_leaf(c)) {
                node.meta[i] = (uint8_t)(((c.count - 1) << 5) | toff);
                for (uint32_t k = 0; k < c.count; k++) out.leaf_tris.push_back(ids[c.first + k]);
                toff += c.count;
            } else {
                node.meta[i] = (uint8_t)ninterior;
                node.imask |= (uint8_t)(1u << i);
                ninterior++;
            }
        }
        quantize(node, cbox, (int)ch.size());
        out.nodes[it.wide] = node;
        // reserve the interior children contiguously, in slot order
        uint32_t base = (uint32_t)out.nodes.size();
        int k = 0;
        for (size_t i = 0; i < ch.size(); i++) {
            if (!is_leaf(bn[ch[i]])) {
                out.nodes.emplace_back();
                q.push_back({ch[i], base + (uint32_t)k});
                k++;
            }
        }
    }
}

}  // namespace rtb
