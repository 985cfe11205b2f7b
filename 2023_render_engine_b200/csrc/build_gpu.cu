// Device build of the acceleration structures (rt_scene_commit with RT_BUILD_DEVICE): the
// reference-order tree and the PLOC 8-wide BVH of the host builders (ref_tree.cpp,
// bvh8_build.cpp), the same bytes, built on the GPU.
//
//   1. scene box and margin: a block reduction of the vertices (min, max and |x| are exact in
//      any order), finished on the host;
//   2. reference-order tree: the Morton keys (code << 32 | triangle id) of ref_sort_key,
//      sorted by a CUB radix sort; interior boxes and leaf counts level by level (interior
//      node i of the FIFO pairing has children 2(i - n) and 2(i - n) + 1, so once the nodes
//      below d are done, every node below n + d/2 can be); each triangle's rank in the static
//      traversal order from the subtree leaf counts, top down;
//   3. PLOC: per round, each cluster's nearest neighbour in the window, the mutual pairs merged
//      by the lower index, new nodes numbered and survivors compacted by one prefix sum
//      (merges in the low word, survivors in the high word);
//   4. depth-first numbering (subtree sizes in creation order, range starts in reverse) and
//      the SAH leaf rule;
//   5. collapse to 8-wide nodes one breadth-first level at a time: a prefix sum over the
//      level's interior-child and leaf-triangle counts gives every node the child_base and
//      tri_base the host's queue gives it;
//   6. triangle records (vertices, rank, id) and the id -> record map.
// Each round or level reads its totals back to the host (8 bytes) to size the next launch.
#include <cub/cub.cuh>

#include <vector>

#include "bvh_common.cuh"
#include "rt_internal.h"

namespace rtb {
namespace {

constexpr int kT = 256;

unsigned blocks_for(uint64_t n) { return (unsigned)std::max<uint64_t>(1, (n + kT - 1) / kT); }

// ------------------------------------------------------------------------------- bounds

constexpr int kBoundBlocks = 1024;

// Per block: min and max per axis of every vertex, both starting at the origin (the
// reference's scene bound starts from the degenerate box at the origin), and max |x|.
__global__ void __launch_bounds__(kT) k_bounds(const float *__restrict__ tri, uint32_t n, float *__restrict__ part)
{
    __shared__ float sm[7][kT];
    float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f}, ma = 0.f;
    for (uint64_t t = blockIdx.x * (uint64_t)kT + threadIdx.x; t < n; t += (uint64_t)gridDim.x * kT) {
        const float *p = tri + 9 * t;
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float x = p[3 * k + c];
                lo[c] = fminf(lo[c], x);
                hi[c] = fmaxf(hi[c], x);
                ma = bv_max(ma, fabsf(x));
            }
    }
    for (int c = 0; c < 3; c++) {
        sm[c][threadIdx.x] = lo[c];
        sm[3 + c][threadIdx.x] = hi[c];
    }
    sm[6][threadIdx.x] = ma;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            for (int c = 0; c < 3; c++) {
                sm[c][threadIdx.x] = fminf(sm[c][threadIdx.x], sm[c][threadIdx.x + s]);
                sm[3 + c][threadIdx.x] = fmaxf(sm[3 + c][threadIdx.x], sm[3 + c][threadIdx.x + s]);
            }
            sm[6][threadIdx.x] = bv_max(sm[6][threadIdx.x], sm[6][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 7) part[7 * blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

// ------------------------------------------------------------------ reference-order tree

struct Frame {
    float lo[3], diag[3];
};

__global__ void k_keys(const float *__restrict__ tri, uint32_t n, Frame f, uint64_t *__restrict__ keys)
{
    const uint32_t t = blockIdx.x * kT + threadIdx.x;
    if (t < n) keys[t] = ref_sort_key(tri + 9 * (size_t)t, t, f.lo, f.diag);
}

__global__ void k_unpack(const uint64_t *__restrict__ keys, uint32_t n, uint32_t *__restrict__ sorted,
                         uint32_t *__restrict__ pos)
{
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = (uint32_t)keys[i];
    sorted[i] = id;
    pos[id] = i;
}

__global__ void k_ref_leaves(const float *__restrict__ tri, const uint32_t *__restrict__ sorted, uint32_t n,
                             float *__restrict__ boxes, uint32_t *__restrict__ cnt)
{
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= n) return;
    const float *p = tri + 9 * (size_t)sorted[i];
    for (int c = 0; c < 3; c++) {
        const float mn = fminf(p[c], p[3 + c]), mx = fmaxf(p[c], p[3 + c]);
        boxes[6 * (size_t)i + c] = fminf(mn, p[6 + c]);
        boxes[6 * (size_t)i + 3 + c] = fmaxf(mx, p[6 + c]);
    }
    cnt[i] = 1;
}

__global__ void k_ref_interior(float *__restrict__ boxes, uint32_t *__restrict__ cnt, uint32_t n, uint32_t b,
                               uint32_t e)
{
    const uint32_t i = b + blockIdx.x * kT + threadIdx.x;
    if (i >= e) return;
    const size_t l = 2 * (size_t)(i - n), r = l + 1;
    for (int c = 0; c < 3; c++) {
        boxes[6 * (size_t)i + c] = fminf(boxes[6 * l + c], boxes[6 * r + c]);
        boxes[6 * (size_t)i + 3 + c] = fmaxf(boxes[6 * l + 3 + c], boxes[6 * r + 3 + c]);
    }
    cnt[i] = cnt[l] + cnt[r];
}

// BVH::intersectRay's static order (BVH.cu:392-445): a popped node ranks its leaf children
// left then right, then its right subtree is walked before its left one.
__global__ void k_ref_rank(const uint32_t *__restrict__ sorted, const uint32_t *__restrict__ cnt, uint32_t n,
                           uint32_t b, uint32_t e, uint32_t *__restrict__ start, uint32_t *__restrict__ rank)
{
    const uint32_t x = b + blockIdx.x * kT + threadIdx.x;
    if (x >= e) return;
    const uint32_t s = start[x];
    const uint32_t l = 2 * (x - n), r = l + 1;
    uint32_t k = 0;
    if (l < n) rank[sorted[l]] = s + k++;
    if (r < n) rank[sorted[r]] = s + k++;
    if (r >= n) start[r] = s + k;
    if (l >= n) start[l] = s + k + (r >= n ? cnt[r] : 0u);
}

// ----------------------------------------------------------------------------------- PLOC

__global__ void k_ploc_leaves(const float *__restrict__ tri, const uint32_t *__restrict__ sorted, uint32_t n,
                              float margin, BBox *__restrict__ bx, uint32_t *__restrict__ cl)
{
    const uint32_t p = blockIdx.x * kT + threadIdx.x;
    if (p >= n) return;
    bx[n - 1 + p] = triangle_box(tri + 9 * (size_t)sorted[p], margin);
    cl[p] = n - 1 + p;
}

__global__ void k_ploc_nn(const BBox *__restrict__ bx, const uint32_t *__restrict__ cl, uint32_t m, uint32_t radius,
                          uint32_t *__restrict__ nn)
{
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= m) return;
    nn[i] = (uint32_t)ploc_nearest(i, m, radius, [&](int64_t j) { return bx[cl[j]]; });
}

// flags: bit 0 (low word) = makes a node (lower index of a mutual pair), bit 32 = survives
__global__ void k_ploc_flags(const uint32_t *__restrict__ nn, uint32_t m, uint64_t *__restrict__ flags)
{
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= m) return;
    const uint32_t j = nn[i];
    const bool mutual = nn[j] == i;
    flags[i] = (uint64_t)(mutual && i < j) | ((uint64_t)(!mutual || i < j) << 32);
}

__global__ void k_ploc_merge(BBox *__restrict__ bx, const uint32_t *__restrict__ cl, const uint32_t *__restrict__ nn,
                             uint32_t m, const uint64_t *__restrict__ flags, const uint64_t *__restrict__ pos,
                             uint32_t made, uint32_t *__restrict__ c0, uint32_t *__restrict__ c1,
                             uint32_t *__restrict__ next, uint64_t *__restrict__ totals)
{
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= m) return;
    const uint64_t f = flags[i], pp = pos[i];
    const uint32_t k = made + (uint32_t)pp;
    if (f & 1u) {
        const uint32_t a = cl[i], b = cl[nn[i]];
        c0[k] = a;
        c1[k] = b;
        BBox u = bx[a];
        bbox_grow(u, bx[b]);
        bx[k] = u;  // a new node: no thread of this merge pass reads it
    }
    if (f >> 32) next[(uint32_t)(pp >> 32)] = (f & 1u) ? k : cl[i];
    if (i == m - 1) *totals = pp + f;
}

// ---------------------------------------------------------- depth-first numbering, leaves

__global__ void k_fill(uint32_t *__restrict__ v, uint64_t n, uint32_t x)
{
    const uint64_t i = (uint64_t)blockIdx.x * kT + threadIdx.x;
    if (i < n) v[i] = x;
}

__global__ void k_sizes(const uint32_t *__restrict__ c0, const uint32_t *__restrict__ c1, uint32_t b, uint32_t e,
                        uint32_t *__restrict__ size)
{
    const uint32_t k = b + blockIdx.x * kT + threadIdx.x;
    if (k < e) size[k] = size[c0[k]] + size[c1[k]];
}

__global__ void k_first(const uint32_t *__restrict__ c0, const uint32_t *__restrict__ c1,
                        const uint32_t *__restrict__ size, uint32_t b, uint32_t e, uint32_t *__restrict__ first)
{
    const uint32_t k = b + blockIdx.x * kT + threadIdx.x;
    if (k >= e) return;
    first[c0[k]] = first[k];
    first[c1[k]] = first[k] + size[c0[k]];
}

__global__ void k_leaf_setup(const uint32_t *__restrict__ sorted, const uint32_t *__restrict__ first,
                             const BBox *__restrict__ bx, const uint32_t *__restrict__ c0,
                             const uint32_t *__restrict__ c1, const uint32_t *__restrict__ size, uint32_t n,
                             uint32_t *__restrict__ ids, uint8_t *__restrict__ leaf)
{
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i < n) {
        ids[first[n - 1 + i]] = sorted[i];
        leaf[n - 1 + i] = 1;
    }
    if (i + 1 < n)
        leaf[i] = sah_leaf(size[i], bbox_area(bx[i]), bbox_area(bx[c0[i]]), size[c0[i]], bbox_area(bx[c1[i]]),
                           size[c1[i]]) ? 1 : 0;
}

// ------------------------------------------------------------------------------ collapse

struct Tree {
    const BBox *bx;
    const uint32_t *c0, *c1, *size, *first, *ids;
    const uint8_t *leaf;
    uint32_t n;
};

__global__ void k_wide_count(Tree tr, const uint32_t *__restrict__ cur, uint32_t ncur, uint32_t *__restrict__ chbuf,
                             uint64_t *__restrict__ counts)
{
    const uint32_t w = blockIdx.x * kT + threadIdx.x;
    if (w >= ncur) return;
    uint32_t ch[8];
    const int nch = wide_children(
        cur[w], ch, [&](uint32_t x) { return tr.leaf[x] != 0; }, [&](uint32_t x, int s) { return s ? tr.c1[x] : tr.c0[x]; },
        [&](uint32_t x) { return bbox_area(tr.bx[x]); });
    uint32_t kint = 0, tcnt = 0;
    for (int i = 0; i < 8; i++) {
        const uint32_t x = i < nch ? ch[i] : 0xFFFFFFFFu;
        chbuf[8 * (size_t)w + i] = x;
        if (i < nch) {
            if (tr.leaf[x])
                tcnt += tr.size[x];
            else
                kint++;
        }
    }
    counts[w] = (uint64_t)kint | ((uint64_t)tcnt << 32);
}

__global__ void k_wide_write(Tree tr, uint32_t ncur, const uint32_t *__restrict__ chbuf,
                             const uint64_t *__restrict__ counts, const uint64_t *__restrict__ offs, uint32_t wstart,
                             uint32_t tstart, Bvh8Node *__restrict__ nodes, uint32_t *__restrict__ leaf_tris,
                             uint32_t *__restrict__ next, uint64_t *__restrict__ totals)
{
    const uint32_t w = blockIdx.x * kT + threadIdx.x;
    if (w >= ncur) return;
    uint32_t ch[8];
    int nch = 0;
    for (int i = 0; i < 8; i++) {
        ch[i] = chbuf[8 * (size_t)w + i];
        if (ch[i] != 0xFFFFFFFFu) nch = i + 1;
    }
    const uint64_t o = offs[w];
    const uint32_t koff = (uint32_t)o, toff = (uint32_t)(o >> 32);
    Bvh8Node node;
    write_wide_node(
        node, ch, nch, wstart + ncur + koff, tstart + toff, [&](uint32_t x) { return tr.leaf[x] != 0; },
        [&](uint32_t x, uint32_t &f, uint32_t &c) {
            f = tr.first[x];
            c = tr.size[x];
        },
        [&](uint32_t x) { return tr.bx[x]; },
        [&](uint32_t rec, uint32_t p) {
            if (rec < tr.n) leaf_tris[rec] = p < tr.n ? tr.ids[p] : 0u;
        },
        [&](uint32_t k, uint32_t x) {
            if (koff + k < tr.n) next[koff + k] = x;
        });
    nodes[wstart + w] = node;
    if (w == ncur - 1) *totals = o + counts[w];
}

__global__ void k_records(const float *__restrict__ tri, const uint32_t *__restrict__ leaf_tris,
                          const uint32_t *__restrict__ rank, const uint8_t *__restrict__ transparent, uint32_t n,
                          TriRecord *__restrict__ recs, uint32_t *__restrict__ leafpos)
{
    const uint32_t r = blockIdx.x * kT + threadIdx.x;
    if (r >= n) return;
    const uint32_t id = min(leaf_tris[r], n - 1);  // every entry is written; the clamp only bounds the read
    const float *p = tri + 9 * (size_t)id;
    TriRecord tr;
    tr.v0 = make_float4(p[0], p[1], p[2], __uint_as_float(rank[id]));
    tr.v1 = make_float4(p[3], p[4], p[5], __uint_as_float(id));
    tr.v2 = make_float4(p[6], p[7], p[8], __uint_as_float(transparent[id] ? 1u : 0u));
    recs[r] = tr;
    leafpos[id] = r;
}

template <class T>
T *buf(DevBuf &b, uint64_t count, int &rc)
{
    if (rc == RT_OK) rc = b.reserve(std::max<uint64_t>(count, 1) * sizeof(T));
    return b.as<T>();
}

}  // namespace

int build_scene_device(rt_scene *s, float margin_out[1])
{
    cudaStream_t st = s->ctx->stream;
    const uint32_t n = (uint32_t)(s->tri9.size() / 9);
    if (n == 0) return fail(RT_ERR_INVALID, "build_scene_device: no triangles");
    DevBuf *B = s->ctx->build;
    DevBuf &d_tri = B[0], &d_part = B[1], &d_keys = B[2], &d_keys2 = B[3], &d_cnt = B[4], &d_start = B[5],
           &d_rank = B[6], &d_bx = B[7], &d_c0 = B[8], &d_c1 = B[9], &d_cl = B[10], &d_cl2 = B[11], &d_nn = B[12],
           &d_flags = B[13], &d_pos = B[14], &d_tot = B[15], &d_size = B[16], &d_first = B[17], &d_ids = B[18],
           &d_leaf = B[19], &d_cur = B[20], &d_next = B[21], &d_chbuf = B[22], &d_counts = B[23], &d_offs = B[24],
           &d_leaf_tris = B[25], &d_tt = B[26], &d_tmp = B[27], &d_tmp2 = B[28], &d_tmp3 = B[29], &d_wide = B[30];
    int rc = RT_OK;
    float *tri = buf<float>(d_tri, 9ull * n, rc);
    RTB_CHECK(rc);
    RTB_CUDA(cudaMemcpyAsync(tri, s->tri9.data(), 36ull * n, cudaMemcpyHostToDevice, st));
    uint8_t *tt = buf<uint8_t>(d_tt, n, rc);
    RTB_CHECK(rc);
    RTB_CUDA(cudaMemcpyAsync(tt, s->tri_transparent.data(), n, cudaMemcpyHostToDevice, st));

    // 1. scene box and margin
    const unsigned nbb = std::min<unsigned>(kBoundBlocks, blocks_for(n));
    float *part = buf<float>(d_part, 7ull * nbb, rc);
    RTB_CHECK(rc);
    k_bounds<<<nbb, kT, 0, st>>>(tri, n, part);
    RTB_CUDA(cudaGetLastError());
    std::vector<float> hp(7ull * nbb);
    RTB_CUDA(cudaMemcpyAsync(hp.data(), part, 28ull * nbb, cudaMemcpyDeviceToHost, st));
    RTB_CUDA(cudaStreamSynchronize(st));
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, maxabs = 0.f;
    for (unsigned b = 0; b < nbb; b++) {
        for (int c = 0; c < 3; c++) {
            lo[c] = fminf(lo[c], hp[7 * b + c]);
            hi[c] = fmaxf(hi[c], hp[7 * b + 3 + c]);
        }
        maxabs = bv_max(maxabs, hp[7 * b + 6]);
    }
    const float margin = std::max(1e-5f * maxabs, 1e-30f);
    margin_out[0] = margin;
    Frame fr;
    for (int c = 0; c < 3; c++) {
        fr.lo[c] = lo[c];
        fr.diag[c] = hi[c] - lo[c];
    }

    // 2. reference-order tree
    uint64_t *keys = buf<uint64_t>(d_keys, n, rc), *keys2 = buf<uint64_t>(d_keys2, n, rc);
    RTB_CHECK(rc);
    k_keys<<<blocks_for(n), kT, 0, st>>>(tri, n, fr, keys);
    size_t tmp_bytes = 0;
    RTB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, keys2, (int)n, 0, 64, st));
    void *tmp = buf<uint8_t>(d_tmp, tmp_bytes, rc);
    RTB_CHECK(rc);
    RTB_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, keys2, (int)n, 0, 64, st));
    RTB_CHECK(s->d_ref_sorted.reserve(4ull * n));
    RTB_CHECK(s->d_ref_pos.reserve(4ull * n));
    RTB_CHECK(s->d_ref_boxes.reserve(24ull * (2ull * n - 1)));
    uint32_t *sorted = s->d_ref_sorted.as<uint32_t>();
    float *rboxes = s->d_ref_boxes.as<float>();
    k_unpack<<<blocks_for(n), kT, 0, st>>>(keys2, n, sorted, s->d_ref_pos.as<uint32_t>());
    uint32_t *cnt = buf<uint32_t>(d_cnt, 2ull * n, rc), *start = buf<uint32_t>(d_start, 2ull * n, rc),
             *rank = buf<uint32_t>(d_rank, n, rc);
    RTB_CHECK(rc);
    k_ref_leaves<<<blocks_for(n), kT, 0, st>>>(tri, sorted, n, rboxes, cnt);
    std::vector<std::pair<uint32_t, uint32_t>> waves;
    for (uint64_t d = n; d + 1 < 2ull * n;) {
        const uint64_t d2 = n + d / 2;
        waves.push_back({(uint32_t)d, (uint32_t)d2});
        k_ref_interior<<<blocks_for(d2 - d), kT, 0, st>>>(rboxes, cnt, n, (uint32_t)d, (uint32_t)d2);
        d = d2;
    }
    RTB_CUDA(cudaMemsetAsync(start, 0, 8ull * n, st));
    RTB_CUDA(cudaMemsetAsync(rank, 0, 4ull * n, st));
    for (auto it = waves.rbegin(); it != waves.rend(); ++it)
        k_ref_rank<<<blocks_for(it->second - it->first), kT, 0, st>>>(sorted, cnt, n, it->first, it->second, start,
                                                                        rank);
    RTB_CUDA(cudaGetLastError());

    // 3. PLOC
    const uint64_t nb = 2ull * n - 1;
    BBox *bx = buf<BBox>(d_bx, nb, rc);
    uint32_t *c0 = buf<uint32_t>(d_c0, n, rc), *c1 = buf<uint32_t>(d_c1, n, rc), *cl = buf<uint32_t>(d_cl, n, rc),
             *cl2 = buf<uint32_t>(d_cl2, n, rc), *nn = buf<uint32_t>(d_nn, n, rc);
    uint64_t *flags = buf<uint64_t>(d_flags, n, rc), *pos = buf<uint64_t>(d_pos, n, rc),
             *tot = buf<uint64_t>(d_tot, 2, rc);
    RTB_CHECK(rc);
    k_ploc_leaves<<<blocks_for(n), kT, 0, st>>>(tri, sorted, n, margin, bx, cl);
    tmp_bytes = 0;
    RTB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flags, pos, (int)n, st));
    tmp = buf<uint8_t>(d_tmp2, tmp_bytes, rc);
    RTB_CHECK(rc);
    std::vector<uint32_t> batches{0};  // internal nodes made per round: [batches[t], batches[t + 1])
    uint32_t m = n, made = 0;
    for (uint32_t round = 0; m > 1; round++) {
        if (round > n) return fail(RT_ERR_TIMEOUT, "build_scene_device: clustering made no progress");
        k_ploc_nn<<<blocks_for(m), kT, 0, st>>>(bx, cl, m, kPlocRadius, nn);
        k_ploc_flags<<<blocks_for(m), kT, 0, st>>>(nn, m, flags);
        RTB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flags, pos, (int)m, st));
        k_ploc_merge<<<blocks_for(m), kT, 0, st>>>(bx, cl, nn, m, flags, pos, made, c0, c1, cl2, tot);
        RTB_CUDA(cudaGetLastError());
        uint64_t t = 0;
        RTB_CUDA(cudaMemcpyAsync(&t, tot, 8, cudaMemcpyDeviceToHost, st));
        RTB_CUDA(cudaStreamSynchronize(st));
        const uint32_t merges = (uint32_t)t, keep = (uint32_t)(t >> 32);
        if (merges == 0 || keep + merges != m) return fail(RT_ERR_TIMEOUT, "build_scene_device: clustering stalled");
        made += merges;
        batches.push_back(made);
        m = keep;
        std::swap(cl, cl2);
    }
    uint32_t root = 0;
    RTB_CUDA(cudaMemcpyAsync(&root, cl, 4, cudaMemcpyDeviceToHost, st));

    // 4. depth-first numbering and leaves
    uint32_t *size = buf<uint32_t>(d_size, nb, rc), *first = buf<uint32_t>(d_first, nb, rc),
             *ids = buf<uint32_t>(d_ids, n, rc);
    uint8_t *leaf = buf<uint8_t>(d_leaf, nb, rc);
    RTB_CHECK(rc);
    RTB_CUDA(cudaMemsetAsync(ids, 0, 4ull * n, st));
    {
        k_fill<<<blocks_for(nb), kT, 0, st>>>(size, nb, 1u);  // leaf sizes; internal sizes overwritten below
        RTB_CUDA(cudaMemsetAsync(first, 0, 4ull * nb, st));
        for (size_t t = 0; t + 1 < batches.size(); t++)
            k_sizes<<<blocks_for(batches[t + 1] - batches[t]), kT, 0, st>>>(c0, c1, batches[t], batches[t + 1],
                                                                            size);
        for (size_t t = batches.size() - 1; t > 0; t--)
            k_first<<<blocks_for(batches[t] - batches[t - 1]), kT, 0, st>>>(c0, c1, size, batches[t - 1],
                                                                             batches[t], first);
        k_leaf_setup<<<blocks_for(n), kT, 0, st>>>(sorted, first, bx, c0, c1, size, n, ids, leaf);
        RTB_CUDA(cudaGetLastError());
    }

    // 5. collapse, level by level
    Bvh8Node *nodes = buf<Bvh8Node>(d_wide, n, rc);  // room for the most nodes n triangles can need
    uint32_t *leaf_tris = buf<uint32_t>(d_leaf_tris, n, rc), *cur = buf<uint32_t>(d_cur, n, rc),
             *next = buf<uint32_t>(d_next, n, rc), *chbuf = buf<uint32_t>(d_chbuf, 8ull * n, rc);
    uint64_t *counts = buf<uint64_t>(d_counts, n, rc), *offs = buf<uint64_t>(d_offs, n, rc);
    RTB_CHECK(rc);
    tmp_bytes = 0;
    RTB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, offs, (int)n, st));
    tmp = buf<uint8_t>(d_tmp3, tmp_bytes, rc);
    RTB_CHECK(rc);
    RTB_CUDA(cudaMemcpyAsync(cur, &root, 4, cudaMemcpyHostToDevice, st));
    RTB_CUDA(cudaMemsetAsync(leaf_tris, 0, 4ull * n, st));
    const Tree tr{bx, c0, c1, size, first, ids, leaf, n};
    uint32_t ncur = 1, wstart = 0, tstart = 0;
    while (ncur > 0) {
        if ((uint64_t)wstart + ncur > n) return fail(RT_ERR_CAPACITY, "build_scene_device: node count overflow");
        k_wide_count<<<blocks_for(ncur), kT, 0, st>>>(tr, cur, ncur, chbuf, counts);
        RTB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, offs, (int)ncur, st));
        k_wide_write<<<blocks_for(ncur), kT, 0, st>>>(tr, ncur, chbuf, counts, offs, wstart, tstart, nodes, leaf_tris,
                                                      next, tot);
        RTB_CUDA(cudaGetLastError());
        uint64_t t = 0;
        RTB_CUDA(cudaMemcpyAsync(&t, tot, 8, cudaMemcpyDeviceToHost, st));
        RTB_CUDA(cudaStreamSynchronize(st));
        wstart += ncur;
        tstart += (uint32_t)(t >> 32);
        ncur = (uint32_t)t;
        std::swap(cur, next);
    }
    if (tstart != n) return fail(RT_ERR_STATE, "build_scene_device: leaf triangles lost");
    s->nnodes = wstart;
    RTB_CHECK(s->d_nodes.reserve(sizeof(Bvh8Node) * (uint64_t)wstart));
    RTB_CUDA(cudaMemcpyAsync(s->d_nodes.ptr, nodes, sizeof(Bvh8Node) * (uint64_t)wstart, cudaMemcpyDeviceToDevice, st));

    // 6. records
    RTB_CHECK(s->d_tris.reserve(sizeof(TriRecord) * (uint64_t)n));
    RTB_CHECK(s->d_leafpos.reserve(4ull * n));
    k_records<<<blocks_for(n), kT, 0, st>>>(tri, leaf_tris, rank, tt, n, s->d_tris.as<TriRecord>(),
                                            s->d_leafpos.as<uint32_t>());
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaStreamSynchronize(st));
    return RT_OK;
}

namespace {

// Shadow-ray transparency of every record (bit 0 of v2.w): the triangle's own flag or its
// material's RT_MATF_TRANSPARENT (Triangle.cu:439-440).
__global__ void k_record_flags(TriRecord *__restrict__ recs, uint32_t n, const uint8_t *__restrict__ tri_transparent,
                               const uint32_t *__restrict__ tri_mat, const uint8_t *__restrict__ mat_transparent,
                               uint32_t nmat)
{
    const uint32_t r = blockIdx.x * kT + threadIdx.x;
    if (r >= n) return;
    const uint32_t id = __float_as_uint(recs[r].v1.w);
    const uint32_t m = tri_mat[id];
    recs[r].v2.w = __uint_as_float((tri_transparent[id] || (m < nmat && mat_transparent[m])) ? 1u : 0u);
}

}  // namespace

int refresh_record_flags(rt_scene *s)
{
    const uint32_t n = (uint32_t)(s->tri9.size() / 9);
    if (n == 0 || !s->d_tris.ptr) return RT_OK;
    cudaStream_t st = s->ctx->stream;
    std::vector<uint8_t> mt(std::max<size_t>(s->materials.size(), 1), 0);
    for (size_t m = 0; m < s->materials.size(); m++) mt[m] = (s->materials[m].flags & RT_MATF_TRANSPARENT) ? 1 : 0;
    RTB_CHECK(s->d_tri_transp.upload(s->tri_transparent.data(), n, st));
    RTB_CHECK(s->d_tri_mat.upload(s->tri_material.data(), 4ull * n, st));
    RTB_CHECK(s->d_mat_transp.upload(mt.data(), mt.size(), st));
    k_record_flags<<<blocks_for(n), kT, 0, st>>>(s->d_tris.as<TriRecord>(), n, s->d_tri_transp.as<uint8_t>(),
                                                 s->d_tri_mat.as<uint32_t>(), s->d_mat_transp.as<uint8_t>(),
                                                 (uint32_t)s->materials.size());
    RTB_CUDA(cudaGetLastError());
    return RT_OK;
}

}  // namespace rtb
