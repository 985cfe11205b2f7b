// Path-guide network: training on the tensor cores and the rt_guide_* entry points.
//
// One training step on B samples (rows padded to a multiple of 128), all contractions on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM):
//   k_guide_wsum      partial sums of the sample weights (their mean normalises the loss)
//   k_guide_train_tc  per 128-row tile: encode, forward, loss gradient per row, backward
//                     through the 5 layers; writes every layer's input and output gradient
//                     feature-major, so the weight gradient is a contraction over rows
//   k_guide_wgrad_tc  dW_l = X_l^T G_l per chunk of rows (FP32 partials), all layers at once
//   k_guide_bias_grad db_l = sum G_l per chunk of rows
//   k_guide_reduce    sum of the chunk partials in a fixed order (deterministic gradient)
//   k_guide_adam      Adam on the FP32 master weights; refreshes the FP16 image
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "guide.cuh"
#include "rt_internal.h"

namespace rtb {

namespace {

constexpr int kWsumBlocks = 128;
constexpr float kAdamB1 = 0.9f, kAdamB2 = 0.99f, kAdamEps = 1e-8f;

__device__ __forceinline__ uint32_t pack_h2(__half a, __half b)
{
    __half2 h = __halves2half2(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

struct TrainArgs {
    const float *q, *dir, *pdf, *w;
    uint64_t B, Bpad;
    __half *xt, *gt;
    float *scal;          // [1] loss sum (accumulated)
    const double *wpart;  // kWsumBlocks partial sums of the weights
    GuideBox box;
};

// ------------------------------------------------------------------ training on tcgen05
//
// k_guide_train_tc: the forward and backward passes of 128-row tiles on the 5th-generation tensor
// cores, two independent 128-thread groups per CTA sharing one copy of the weights in shared
// memory. Per layer one thread issues tcgen05.mma (M = 128 rows, FP16 operands in K-major core
// matrices, FP32 accumulator in the group's 64 TMEM columns) and commits to the group's
// mbarrier; every thread then reads its own row back (tcgen05.ld), applies bias and ReLU (forward)
// or the ReLU mask (backward) and writes the next operand. The forward operand is W_l^T (the
// inference staging); the backward operand is W_l itself, restaged once per CTA. Each thread
// keeps its row's ReLU signs as bit masks, so only two operand buffers per group are needed.
// Every layer input X_l and output gradient G_l is also written feature-major (planes of Bp rows)
// for the weight gradient.
constexpr int kFbGroups = 2;
constexpr int kFbWb = 50432;  // backward weights W_1..W_4 (64 rows of out_l halves), 8 KB slots
__host__ __device__ constexpr int fb_wb(int l) { return kFbWb + (l - 1) * 8192; }
constexpr int kFbGroup0 = kFbWb + 4 * 8192;
constexpr int kFbBufA = 128 * kGuideIn * 2;  // X_0 (144 halves per row); later X_2, X_4, G_3, G_1
constexpr int kFbBufB = 128 * 64 * 2;        // X_1, X_3, G_4, G_2
constexpr int kFbGroupBytes = kFbBufA + kFbBufB;
constexpr int kFbBar = kFbGroup0 + kFbGroups * kFbGroupBytes;
constexpr int kFbSmem = kFbBar + 8 * kFbGroups + 16;
constexpr int kFbTmemCols = 64 * kFbGroups;
static_assert(kTcBias + 4 * (4 * 64 + 48) <= kFbWb && kFbGroup0 % 128 == 0 && kFbBar % 8 == 0, "train layout");
static_assert(kFbSmem <= 227 * 1024, "training shared memory");

// one M = 128 pass of layer operands: D[tmem] = A (kc_a chunks per row) * B^T over `ksteps`
// K = 16 steps, issued by the calling thread and committed to `bar`
__device__ __forceinline__ void fb_mma(uint32_t tmem, uint32_t a0, uint32_t kca, uint32_t b0, uint32_t kcb, int ksteps,
                                       int n, uint64_t *bar)
{
    const uint32_t idesc = umma_idesc_f16(128, n);
    for (int s = 0; s < ksteps; s++)
        umma_f16(tmem, umma_desc(a0 + 256u * s, 128u, 128u * kca), umma_desc(b0 + 256u * s, 128u, 128u * kcb), idesc,
                 s > 0 ? 1u : 0u);
    umma_commit(bar);
}

// The group's 128-row operand tile (kc chunks of 8 halves per row, core-matrix layout) to the
// feature-major planes dst[f * Bp + row0 + r] for features f < nfeat: each 16-byte store holds
// one feature of 8 consecutive rows (read from the 8 rows of one core matrix).
__device__ __forceinline__ void tile_to_planes(const unsigned char *tile, int kc, int nfeat, __half *dst, uint64_t Bp,
                                               uint64_t row0, int gt)
{
    for (int i = gt; i < nfeat * 16; i += 128) {
        const int f = i >> 4, rg = i & 15;  // feature, group of 8 rows
        const unsigned char *src = tile + tc_chunk((uint32_t)(8 * rg), (uint32_t)(f >> 3), (uint32_t)kc) + 2 * (f & 7);
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const __half lo = *reinterpret_cast<const __half *>(src + 32 * j);
            const __half hi = *reinterpret_cast<const __half *>(src + 32 * j + 16);
            w[j] = pack_h2(lo, hi);
        }
        *reinterpret_cast<uint4 *>(dst + (uint64_t)f * Bp + row0 + 8 * rg) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

__global__ void __launch_bounds__(128 * kFbGroups, 1) k_guide_train_tc(const uint4 *img, TrainArgs A)
{
    extern __shared__ __align__(128) unsigned char fb_smem[];
    unsigned char *sm = fb_smem;
    __shared__ double wsum;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = tid >> 7, gt = tid & 127;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kFbBar) + grp;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kFbBar + 8 * kFbGroups);
    const unsigned char *ib = reinterpret_cast<const unsigned char *>(img);
    // forward weights (W_l^T) and biases, as the inference kernel stages them
#pragma unroll 1
    for (int l = 0; l < kGuideLayers; l++) {
        const int kc = guide_in(l) / 8, nrows = guide_out(l);
        for (int i = tid; i < nrows * kc; i += blockDim.x) {
            const int r = i / kc, c = i - r * kc;
            *reinterpret_cast<uint4 *>(sm + tc_w(l) + tc_chunk(r, c, kc)) =
                *reinterpret_cast<const uint4 *>(ib + 2 * (guide_iw(l) + r * guide_stride(l)) + 16 * c);
        }
    }
    for (int i = tid; i < (4 * 64 + 48) / 4; i += blockDim.x)
        reinterpret_cast<uint4 *>(sm + kTcBias)[i] = reinterpret_cast<const uint4 *>(ib + kGuideImgBias)[i];
    // backward weights W_l (l = 1..4): row i (input), chunk c = outputs 8c .. 8c + 7
    const __half *ih = reinterpret_cast<const __half *>(img);
#pragma unroll 1
    for (int l = 1; l < kGuideLayers; l++) {
        const int kc = guide_out(l) / 8;
        for (int i = tid; i < 64 * kc; i += blockDim.x) {
            const int r = i / kc, c = i - r * kc;
            uint32_t w[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const __half lo = ih[guide_iw(l) + (8 * c + 2 * j) * guide_stride(l) + r];
                const __half hi = ih[guide_iw(l) + (8 * c + 2 * j + 1) * guide_stride(l) + r];
                w[j] = pack_h2(lo, hi);
            }
            *reinterpret_cast<uint4 *>(sm + fb_wb(l) + tc_chunk(r, c, kc)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    if (tid < 32) {
        double sw = 0.0;
        for (int i = tid; i < kWsumBlocks; i += 32) sw += A.wpart[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sw += __shfl_xor_sync(0xffffffffu, sw, o);
        if (tid == 0) wsum = sw;
    }
    if (gt == 0) mbar_init(bar, 1);
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, kFbTmemCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot + (uint32_t)(64 * grp);
    const uint32_t tlane = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const uint32_t bar_id = 1u + (uint32_t)grp;
    const float *bias = reinterpret_cast<const float *>(sm + kTcBias);
    unsigned char *bufA = sm + kFbGroup0 + grp * kFbGroupBytes, *bufB = bufA + kFbBufA;
    const uint32_t aA = smem_u32(bufA), aB = smem_u32(bufB);
    const float wmean = A.B ? (float)(wsum / (double)A.B) : 0.f;
    const float winv = wmean > 0.f ? 1.f / wmean : 0.f;
    const uint64_t Bp = A.Bpad;
    float lsum = 0.f;
    uint32_t phase = 0;
    bool failed = false;
    // waits for this group's MMA batch; false (for the whole group) when a wait ran out
    auto wait_mma = [&]() -> bool {
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar, phase, kUmmaWaitPolls));
        phase ^= 1u;
        tc_fence_after();
        return !group_sync_or(bar_id, !ok);
    };
    // the operand just written becomes visible to the tensor core; thread 0 of the group issues,
    // then the group copies the operand to its feature-major planes while the MMA runs
    auto issue = [&](uint32_t a0, uint32_t kca, uint32_t b0, uint32_t kcb, int ksteps, int n, const unsigned char *tile,
                     int nfeat, __half *planes, uint64_t row0) {
        fence_async_smem();
        tc_fence_before();
        group_sync_or(bar_id, false);
        if (gt == 0) {
            tc_fence_after();
            fb_mma(tmem, a0, kca, b0, kcb, ksteps, n, bar);
        }
        tile_to_planes(tile, (int)kca, nfeat, planes, Bp, row0, gt);
    };
    const uint32_t stride = gridDim.x * kFbGroups;
    for (uint64_t tile = (uint64_t)blockIdx.x * kFbGroups + grp; !failed && tile * 128 < Bp; tile += stride) {
        const uint64_t row = tile * 128 + gt;
        const bool in_b = row < A.B, in_p = row < Bp;
        float q[9];
#pragma unroll
        for (int i = 0; i < 9; i++) q[i] = in_b ? A.q[9 * row + i] : 0.f;
        {
            __half2 e[72];
            guide_encode(0, q, A.box, e);
            guide_encode(1, q, A.box, e);
#pragma unroll
            for (int c = 0; c < kGuideIn / 8; c++)
                *reinterpret_cast<uint4 *>(bufA + tc_chunk(gt, c, kGuideIn / 8)) =
                    *reinterpret_cast<const uint4 *>(&e[4 * c]);
        }
        const uint64_t row0 = tile * 128;
        // forward: X_0 (A) -> X_1 (B) -> X_2 (A) -> X_3 (B) -> X_4 (A) -> outputs
        uint32_t mask[4][2];
#pragma unroll 1
        for (int l = 0; l < kGuideLayers - 1 && !failed; l++) {
            const uint32_t src = (l & 1) ? aB : aA;
            unsigned char *dst = (l & 1) ? bufA : bufB;
            issue(src, guide_in(l) / 8, smem_u32(sm + tc_w(l)), guide_in(l) / 8, guide_in(l) / 16, 64,
                  (l & 1) ? bufB : bufA, guide_in(l), A.xt + (uint64_t)guide_xoff(l) * Bp, row0);
            if (!wait_mma()) {
                failed = true;
                break;
            }
            const float *b = bias + guide_ib(l);
            uint32_t m0 = 0, m1 = 0;
#pragma unroll
            for (int h = 0; h < 4; h++) {
                float v[16];
                tmem_ld16(tlane + 16u * h, v);
                uint32_t w[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    w[j] = relu_half2(v[2 * j] + b[16 * h + 2 * j], v[2 * j + 1] + b[16 * h + 2 * j + 1]);
                    const __half2 hv = *reinterpret_cast<const __half2 *>(&w[j]);
                    const uint32_t bits = (__low2float(hv) > 0.f ? 1u : 0u) | (__high2float(hv) > 0.f ? 2u : 0u);
                    const int f = 16 * h + 2 * j;
                    if (f < 32)
                        m0 |= bits << f;
                    else
                        m1 |= bits << (f - 32);
                }
                *reinterpret_cast<uint4 *>(dst + tc_chunk(gt, 2 * h, 8)) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4 *>(dst + tc_chunk(gt, 2 * h + 1, 8)) = make_uint4(w[4], w[5], w[6], w[7]);
            }
            mask[l][0] = m0;
            mask[l][1] = m1;
        }
        if (failed) break;
        issue(aA, 8, smem_u32(sm + tc_w(4)), 8, 4, kGuideOut, bufA, kGuideHidden, A.xt + (uint64_t)guide_xoff(4) * Bp,
              row0);
        if (!wait_mma()) {
            failed = true;
            break;
        }
        {
            float o[kGuideOut];
#pragma unroll
            for (int h = 0; h < kGuideOut / 16; h++) tmem_ld16(tlane + 16u * h, o + 16 * h);
            const float *b = bias + guide_ib(4);
#pragma unroll
            for (int j = 0; j < kGuideOut; j++) o[j] += b[j];
            float dout[kGuideOut];
            if (in_b) {
                const float wt = fminf(A.w[row] * winv, kGuideWeightClip);
                const V3 wi = v3(A.dir[3 * row], A.dir[3 * row + 1], A.dir[3 * row + 2]);
                lsum += guide_loss_grad(o, wi, A.pdf[row], wt, dout);
            } else {
#pragma unroll
                for (int j = 0; j < kGuideOut; j++) dout[j] = 0.f;
            }
            uint32_t w[kGuideOut / 2];
#pragma unroll
            for (int j = 0; j < kGuideOut / 2; j++) {
                const __half2 hv =
                    __floats2half2_rn(dout[2 * j] * (1.f / kGuideGradScale), dout[2 * j + 1] * (1.f / kGuideGradScale));
                w[j] = *reinterpret_cast<const uint32_t *>(&hv);
            }
#pragma unroll
            for (int c = 0; c < kGuideOut / 8; c++)
                *reinterpret_cast<uint4 *>(bufB + tc_chunk(gt, c, kGuideOut / 8)) =
                    make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
        }
        // backward: G_4 (B) -> G_3 (A) -> G_2 (B) -> G_1 (A) -> G_0 (planes only)
#pragma unroll 1
        for (int l = kGuideLayers - 1; l >= 1 && !failed; l--) {
            const uint32_t src = (l & 1) ? aA : aB;  // l = 4: G_4 in B; 3: G_3 in A; ...
            unsigned char *dst = (l & 1) ? bufB : bufA;
            const int kco = guide_out(l) / 8;
            issue(src, kco, smem_u32(sm + fb_wb(l)), kco, guide_out(l) / 16, 64, (l & 1) ? bufA : bufB, guide_out(l),
                  A.gt + (uint64_t)guide_goff(l) * Bp, row0);
            if (!wait_mma()) {
                failed = true;
                break;
            }
            const uint32_t m0 = mask[l - 1][0], m1 = mask[l - 1][1];
#pragma unroll
            for (int h = 0; h < 4; h++) {
                float v[16];
                tmem_ld16(tlane + 16u * h, v);
                uint32_t w[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int f = 16 * h + 2 * j;
                    const uint32_t bits = f < 32 ? (m0 >> f) : (m1 >> (f - 32));
                    const __half2 hv = __floats2half2_rn((bits & 1u) ? v[2 * j] : 0.f, (bits & 2u) ? v[2 * j + 1] : 0.f);
                    w[j] = *reinterpret_cast<const uint32_t *>(&hv);
                }
                *reinterpret_cast<uint4 *>(dst + tc_chunk(gt, 2 * h, 8)) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4 *>(dst + tc_chunk(gt, 2 * h + 1, 8)) = make_uint4(w[4], w[5], w[6], w[7]);
            }
            if (l == 1) {  // G_0 feeds no further product: only its planes
                group_sync_or(bar_id, false);
                tile_to_planes(dst, 8, kGuideHidden, A.gt, Bp, row0, gt);
            }
        }
    }
    if (failed) {
        if (gt == 0) atomicOr(reinterpret_cast<uint32_t *>(A.scal) + 2, 2u);  // tensor-core wait ran out
        mbar_wait_bounded(bar, phase ^ 1u, kUmmaWaitPolls);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0 && lsum != 0.f) atomicAdd(A.scal + 1, lsum);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        __syncwarp();
        tmem_dealloc(*tslot, kFbTmemCols);
    }
}

// k_guide_wgrad_tc: dW_l^T = G_l^T X_l over a chunk of rows, all five layers, on tcgen05. The
// feature-major planes are K-major operands with the rows as K: A = G_l^T (M = 128 lanes, the
// out_l valid ones first; the rest of the tile is the next layer's rows or unused bytes, whose
// products land in TMEM lanes nobody reads), B = X_l^T (N = in_l). Stages of 64 rows are loaded
// into one of two shared-memory buffers while the tensor core works on the other; the five
// accumulators (144 + 4 x 64 TMEM columns) stay in TMEM for the whole chunk, which then writes
// its FP32 partial dW in the master layout.
// rows per CTA: a multiple of 64 chosen per step so the chunks about cover the SMs once
__host__ __device__ inline uint64_t wgrad_chunk(uint64_t Bp, uint32_t sms)
{
    const uint64_t c = (Bp / (sms ? sms : 1) + 63) / 64 * 64;
    return c < 256 ? 256 : c;
}
constexpr int kWgStageA = 5 * 8192 + 8192;         // G^T tiles: layer l at l * 8 KB (64 valid rows)
constexpr int kWgStageB = 18 * 1024 + 4 * 8192;    // X^T tiles: layer 0 (144 rows), layers 1-4 (64)
constexpr int kWgStage = kWgStageA + kWgStageB;
constexpr int kWgBar = 2 * kWgStage;
constexpr int kWgSmem = kWgBar + 16 + 16;
constexpr int kWgTmemCols = 512;
static_assert(kWgSmem <= 227 * 1024, "weight-gradient shared memory");
__host__ __device__ constexpr int wg_b(int l) { return kWgStageA + (l == 0 ? 0 : 18 * 1024 + (l - 1) * 8192); }
__host__ __device__ constexpr int wg_col(int l) { return l == 0 ? 0 : kGuideIn + (l - 1) * 64; }

__global__ void __launch_bounds__(128, 1) k_guide_wgrad_tc(const __half *xt, const __half *gt, uint64_t Bp,
                                                           uint64_t chunk, float *partial, float *scal)
{
    extern __shared__ __align__(128) unsigned char wg_smem[];
    unsigned char *sm = wg_smem;
    const int tid = threadIdx.x, warp = tid >> 5;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kWgBar);  // one per buffer
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kWgBar + 16);
    const uint64_t r0 = (uint64_t)blockIdx.x * chunk;
    const uint64_t r1 = r0 + chunk < Bp ? r0 + chunk : Bp;
    const int nstages = (int)((r1 - r0) / 64);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, kWgTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    uint32_t phase[2] = {0u, 0u};
    bool failed = false;
    for (int s = 0; s < nstages && !failed; s++) {
        const int b = s & 1;
        unsigned char *buf = sm + b * kWgStage;
        if (s >= 2) {  // the MMAs of stage s - 2 read this buffer
            const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar + b, phase[b], kUmmaWaitPolls));
            phase[b] ^= 1u;
            failed = __syncthreads_or(!ok) != 0;
            if (failed) break;
        }
        const uint64_t rs = r0 + 64ull * s;
        // G^T: 304 features x 8 chunks of 8 rows; X^T: 400 features x 8 chunks
        for (int i = tid; i < kGuideGFeatures * 8; i += 128) {
            const int f = i >> 3, c = i & 7;
            const int l = f < 4 * kGuideHidden ? f / kGuideHidden : 4, fl = f - guide_goff(l);
            *reinterpret_cast<uint4 *>(buf + l * 8192 + tc_chunk(fl, c, 8)) =
                __ldg(reinterpret_cast<const uint4 *>(gt + (uint64_t)f * Bp + rs) + c);
        }
        for (int i = tid; i < kGuideXFeatures * 8; i += 128) {
            const int f = i >> 3, c = i & 7;
            const int l = f < kGuideIn ? 0 : 1 + (f - kGuideIn) / kGuideHidden, fl = f - guide_xoff(l);
            *reinterpret_cast<uint4 *>(buf + wg_b(l) + tc_chunk(fl, c, 8)) =
                __ldg(reinterpret_cast<const uint4 *>(xt + (uint64_t)f * Bp + rs) + c);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t base = smem_u32(buf);
#pragma unroll 1
            for (int l = 0; l < kGuideLayers; l++) {
                const uint32_t idesc = umma_idesc_f16(128, guide_in(l));
                for (int k = 0; k < 4; k++)
                    umma_f16(tmem + (uint32_t)wg_col(l), umma_desc(base + l * 8192 + 256u * k, 128u, 1024u),
                             umma_desc(base + wg_b(l) + 256u * k, 128u, 1024u), idesc, (s > 0 || k > 0) ? 1u : 0u);
            }
            umma_commit(bar + b);
        }
    }
    // the last batch of each buffer
    for (int b = 0; b < 2 && !failed; b++) {
        const int last = nstages - 1 - ((nstages - 1 - b) & 1);  // latest stage that used buffer b
        if (last < 0 || last < nstages - 2) continue;
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar + b, phase[b], kUmmaWaitPolls));
        phase[b] ^= 1u;
        failed = __syncthreads_or(!ok) != 0;
    }
    tc_fence_after();
    float *part = partial + (uint64_t)blockIdx.x * kGuideParamCount;
    if (!failed && warp < 2) {  // TMEM lanes 0..63: the output features
        const int o = 32 * warp + (tid & 31);
        const uint32_t tl = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll 1
        for (int l = 0; l < kGuideLayers; l++) {
            const int nin = guide_in(l), out = guide_out(l);
            for (int c0 = 0; c0 < nin; c0 += 16) {
                float v[16];
                tmem_ld16(tl + (uint32_t)(wg_col(l) + c0), v);
                if (o < out)
#pragma unroll
                    for (int j = 0; j < 16; j++) part[guide_pw(l) + (c0 + j) * out + o] = v[j];
            }
        }
    }
    if (failed) {
        if (tid == 0) atomicOr(reinterpret_cast<uint32_t *>(scal) + 2, 2u);
        for (int b = 0; b < 2; b++) mbar_wait_bounded(bar + b, phase[b], kUmmaWaitPolls);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        __syncwarp();
        tmem_dealloc(tmem, kWgTmemCols);
    }
}

// db_l = sum of G_l over the chunk's rows (feature-major planes), one warp per 8 features
__global__ void __launch_bounds__(256) k_guide_bias_grad(const __half *gt, uint64_t Bp, uint64_t chunk, float *partial)
{
    const uint64_t r0 = (uint64_t)blockIdx.x * chunk;
    const uint64_t r1 = r0 + chunk < Bp ? r0 + chunk : Bp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *part = partial + (uint64_t)blockIdx.x * kGuideParamCount;
    for (int f = blockIdx.y * 64 + warp; f < kGuideGFeatures && f < (int)blockIdx.y * 64 + 64; f += 8) {
        const uint4 *g4 = reinterpret_cast<const uint4 *>(gt + (uint64_t)f * Bp + r0);
        float s = 0.f;
        for (uint64_t i = lane; i < (r1 - r0) / 8; i += 32) {
            const uint4 v = __ldg(g4 + i);
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float2 h = __half22float2(*reinterpret_cast<const __half2 *>(&w[k]));
                s += h.x + h.y;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const int l = f < 4 * kGuideHidden ? f / kGuideHidden : 4;
            part[guide_pb(l) + (f - guide_goff(l))] = s;
        }
    }
}

// partial sums of the sample weights (double, fixed order); block 0 also clears the loss
// sum and the non-finite flag of this step
__global__ void __launch_bounds__(256) k_guide_wsum(const float *w, uint64_t B, double *part, float *scal)
{
    __shared__ double red[8];
    double s = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < B; i += (uint64_t)kWsumBlocks * 256)
        s += (double)w[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < 8; i++) t += red[i];
        part[blockIdx.x] = t;
        if (blockIdx.x == 0) {
            scal[1] = 0.f;
            reinterpret_cast<uint32_t *>(scal)[2] = 0u;
        }
    }
}

__global__ void k_guide_reduce(const float *partial, uint32_t nchunks, float scale, float *grad, float *scal)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (uint32_t)kGuideParamCount) return;
    float g = 0.f;
    for (uint32_t c = 0; c < nchunks; c++) g += partial[(uint64_t)c * kGuideParamCount + p];
    g *= scale;
    grad[p] = g;
    if (!isfinite(g)) atomicOr(reinterpret_cast<uint32_t *>(scal) + 2, 1u);
}

struct AdamArgs {
    float lr, bc1, bc2;
};

__device__ __forceinline__ void image_write(int p, float w, __half *img_w, float *img_b)
{
    int l = 0;
    while (l < kGuideLayers - 1 && p >= guide_pw(l + 1)) l++;
    if (p < guide_pb(l)) {
        const int i = p - guide_pw(l), out = guide_out(l);
        img_w[guide_iw(l) + (i % out) * guide_stride(l) + i / out] = __float2half_rn(w);
    } else {
        img_b[guide_ib(l) + (p - guide_pb(l))] = w;
    }
}

__global__ void k_guide_adam(const float *grad, const float *scal, float *master, float *m, float *v, __half *img_w,
                             float *img_b, AdamArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kGuideParamCount) return;
    if (reinterpret_cast<const uint32_t *>(scal)[2]) return;  // a non-finite gradient: skip the step
    const float g = grad[p];
    const float mm = kAdamB1 * m[p] + (1.f - kAdamB1) * g;
    const float vv = kAdamB2 * v[p] + (1.f - kAdamB2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float w = master[p] - a.lr * (mm / a.bc1) / (sqrtf(vv / a.bc2) + kAdamEps);
    master[p] = w;
    image_write(p, w, img_w, img_b);
}

// ------------------------------------------------------------------ batched evaluation

// every query row is evaluated (the sinks below see valid = true for each of their rows)
struct QuerySrc {
    const float *q;
    __device__ bool operator()(uint32_t row, float *o) const
    {
#pragma unroll
        for (int i = 0; i < 9; i++) o[i] = q[9ull * row + i];
        return true;
    }
};

struct RawSink {
    float *out;
    __device__ void operator()(uint32_t row, bool valid, const float *o) const
    {
        if (!valid) return;
        for (int i = 0; i < kGuideOut; i++) out[(uint64_t)row * kGuideOut + i] = o[i];
    }
};

struct PdfSink {
    const float *dir, *pdfb;
    float *out;
    __device__ void operator()(uint32_t row, bool valid, const float *o) const
    {
        if (!valid) return;
        GuideParams P;
        guide_decode(o, P);
        const V3 w = v3(dir[3ull * row], dir[3ull * row + 1], dir[3ull * row + 2]);
        out[row] = P.alpha * guide_pdf(P, w) + (1.f - P.alpha) * pdfb[row];
    }
};

struct SampleSink {
    const float *u;
    float *dirs, *pdf;
    __device__ void operator()(uint32_t row, bool valid, const float *o) const
    {
        if (!valid) return;
        GuideParams P;
        guide_decode(o, P);
        const V3 w = guide_sample(P, u[3ull * row], u[3ull * row + 1], u[3ull * row + 2]);
        dirs[3ull * row] = w.x;
        dirs[3ull * row + 1] = w.y;
        dirs[3ull * row + 2] = w.z;
        pdf[row] = guide_pdf(P, w);
    }
};

template <class Sink>
__global__ void __launch_bounds__(kInferWarps * 32, 1) k_guide_eval(const uint4 *img, GuideBox box, uint32_t n,
                                                                  QuerySrc src, Sink sink, uint32_t *werr)
{
    guide_infer_rows(img, box, n, src, sink, werr);
}

// ------------------------------------------------------------------ training samples

// PCG hash (Jarzynski and Olano, "Hash Functions for GPU Rendering", 2020)
__device__ __forceinline__ uint32_t pcg_hash(uint32_t x)
{
    const uint32_t s = x * 747796405u + 2891336453u;
    const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}

__device__ __forceinline__ float record_weight(const GuideRecord &r)
{
    float s = 0.f;
    if (r.d.y > 0.f) s += r.e.x / r.d.y;
    if (r.d.z > 0.f) s += r.e.y / r.d.z;
    if (r.d.w > 0.f) s += r.e.z / r.d.w;
    return s * (1.f / 3.f);
}

__global__ void k_guide_gather(const GuideRecord *recs, const uint32_t *nz, uint32_t nnz, uint32_t B, uint32_t seed,
                               float *q, float *dir, float *pdf, float *w)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const uint32_t h = pcg_hash(i ^ pcg_hash(seed));
    const uint32_t j = (uint32_t)(((uint64_t)h * nnz) >> 32);
    const GuideRecord r = recs[nz[j]];
    const float v[9] = {r.a.x, r.a.y, r.a.z, r.a.w, r.b.x, r.b.y, r.b.z, r.b.w, r.c.x};
#pragma unroll
    for (int k = 0; k < 9; k++) q[9ull * i + k] = v[k];
    dir[3ull * i] = r.c.y;
    dir[3ull * i + 1] = r.c.z;
    dir[3ull * i + 2] = r.c.w;
    pdf[i] = r.d.x;
    w[i] = record_weight(r);
}

}  // namespace

GuideBox guide_box(const rt_guide *g)
{
    GuideBox b;
    const float *lo = g->opts.bbox_min, *hi = g->opts.bbox_max;
    b.lo = make_float3(lo[0], lo[1], lo[2]);
    b.inv_ext = make_float3(1.f / (hi[0] - lo[0]), 1.f / (hi[1] - lo[1]), 1.f / (hi[2] - lo[2]));
    return b;
}

static void build_image(const float *master, std::vector<uint8_t> &img)
{
    img.assign(kGuideImgBytes, 0);
    __half *h = reinterpret_cast<__half *>(img.data());
    float *b = reinterpret_cast<float *>(img.data() + kGuideImgBias);
    for (int l = 0; l < kGuideLayers; l++) {
        const int in = guide_in(l), out = guide_out(l);
        for (int k = 0; k < in; k++)
            for (int n = 0; n < out; n++)
                h[guide_iw(l) + n * guide_stride(l) + k] = __float2half_rn(master[guide_pw(l) + k * out + n]);
        for (int n = 0; n < out; n++) b[guide_ib(l) + n] = master[guide_pb(l) + n];
    }
}

static int guide_upload_params(rt_guide *g, const float *host)
{
    cudaStream_t st = g->ctx->stream;
    std::vector<uint8_t> img;
    build_image(host, img);
    RTB_CHECK(g->master.upload(host, 4ull * kGuideParamCount, st));
    RTB_CHECK(g->img.upload(img.data(), img.size(), st));
    RTB_CHECK(g->adam_m.reserve(4ull * kGuideParamCount));
    RTB_CHECK(g->adam_v.reserve(4ull * kGuideParamCount));
    RTB_CUDA(cudaMemsetAsync(g->adam_m.ptr, 0, 4ull * kGuideParamCount, st));
    RTB_CUDA(cudaMemsetAsync(g->adam_v.ptr, 0, 4ull * kGuideParamCount, st));
    RTB_CUDA(cudaStreamSynchronize(st));  // `img` is pageable host memory
    g->step = 0;
    return RT_OK;
}

// One training step on device arrays (B rows). loss_out / grad_host may be null.
int guide_train(rt_guide *g, const float *q, const float *dir, const float *pdf, const float *w, uint64_t B, int apply,
                float *grad_host, float *loss_out)
{
    cudaStream_t st = g->ctx->stream;
    if (B == 0) {
        if (loss_out) *loss_out = 0.f;
        if (grad_host) std::memset(grad_host, 0, 4ull * kGuideParamCount);
        return RT_OK;
    }
    const uint64_t Bp = (B + 127) / 128 * 128;  // whole 128-row tiles
    const uint64_t chunk = wgrad_chunk(Bp, (uint32_t)std::max(g->ctx->sm_count, 1));
    const uint32_t nchunks = (uint32_t)((Bp + chunk - 1) / chunk);
    RTB_CHECK(g->xt.reserve(2ull * kGuideXFeatures * Bp));
    RTB_CHECK(g->gt.reserve(2ull * kGuideGFeatures * Bp));
    RTB_CHECK(g->partial.reserve(4ull * kGuideParamCount * nchunks));
    RTB_CHECK(g->grad.reserve(4ull * kGuideParamCount));
    RTB_CHECK(g->scal.reserve(64 + 8 * kWsumBlocks));
    if (!g->host_scal) RTB_CUDA(cudaMallocHost(&g->host_scal, 64));
    float *scal = g->scal.as<float>();
    double *wpart = reinterpret_cast<double *>(g->scal.as<uint8_t>() + 64);
    k_guide_wsum<<<kWsumBlocks, 256, 0, st>>>(w, B, wpart, scal);
    RTB_CUDA(cudaGetLastError());
    if (!(device_slot(SLOT_SMEM_ATTRS) & SMEM_GUIDE_TRAIN)) {
        RTB_CUDA(cudaFuncSetAttribute(k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kFbSmem));
        RTB_CUDA(cudaFuncSetAttribute(k_guide_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem));
        or_device_slot(SLOT_SMEM_ATTRS, SMEM_GUIDE_TRAIN);
    }
    TrainArgs a{q, dir, pdf, w, B, Bp, g->xt.as<__half>(), g->gt.as<__half>(), scal, wpart, guide_box(g)};
    const uint64_t tiles = Bp / 128;
    const unsigned grid =
        (unsigned)std::min<uint64_t>((tiles + kFbGroups - 1) / kFbGroups, (uint64_t)std::max(g->ctx->sm_count, 1));
    k_guide_train_tc<<<grid, 128 * kFbGroups, kFbSmem, st>>>(g->img.as<uint4>(), a);
    RTB_CUDA(cudaGetLastError());
    k_guide_wgrad_tc<<<nchunks, 128, kWgSmem, st>>>(g->xt.as<__half>(), g->gt.as<__half>(), Bp, chunk,
                                                    g->partial.as<float>(), scal);
    RTB_CUDA(cudaGetLastError());
    k_guide_bias_grad<<<dim3(nchunks, (kGuideGFeatures + 63) / 64), 256, 0, st>>>(g->gt.as<__half>(), Bp, chunk,
                                                                              g->partial.as<float>());
    RTB_CUDA(cudaGetLastError());
    const unsigned pblocks = (kGuideParamCount + 255) / 256;
    k_guide_reduce<<<pblocks, 256, 0, st>>>(g->partial.as<float>(), nchunks, kGuideGradScale / (float)B,
                                            g->grad.as<float>(), scal);
    RTB_CUDA(cudaGetLastError());
    if (apply) {
        g->step++;
        g->trained = true;
        AdamArgs ad;
        ad.lr = g->opts.learning_rate;
        ad.bc1 = 1.f - (float)std::pow((double)kAdamB1, (double)g->step);
        ad.bc2 = 1.f - (float)std::pow((double)kAdamB2, (double)g->step);
        k_guide_adam<<<pblocks, 256, 0, st>>>(g->grad.as<float>(), scal, g->master.as<float>(), g->adam_m.as<float>(),
                                              g->adam_v.as<float>(), g->img.as<__half>(),
                                              reinterpret_cast<float *>(g->img.as<uint8_t>() + kGuideImgBias), ad);
        RTB_CUDA(cudaGetLastError());
    }
    if (loss_out || grad_host) {
        RTB_CUDA(cudaMemcpyAsync(g->host_scal, scal, 16, cudaMemcpyDeviceToHost, st));
        if (grad_host)
            RTB_CUDA(cudaMemcpyAsync(grad_host, g->grad.ptr, 4ull * kGuideParamCount, cudaMemcpyDeviceToHost, st));
        RTB_CUDA(cudaStreamSynchronize(st));
        if (static_cast<const uint32_t *>(g->host_scal)[2] & 2u)
            return fail(RT_ERR_TIMEOUT, "guide training: a tensor-core completion wait timed out");
        if (loss_out) *loss_out = static_cast<const float *>(g->host_scal)[1] / (float)B;
    }
    return RT_OK;
}

}  // namespace rtb

using namespace rtb;

static int guide_init_params(rt_guide *g);

extern "C" {

int rt_guide_create(rt_context *ctx, const rt_guide_opts *opts, rt_guide **out)
{
    if (!ctx || !opts || !out) return fail(RT_ERR_INVALID, "rt_guide_create: null argument");
    for (int a = 0; a < 3; a++)
        if (!(opts->bbox_max[a] > opts->bbox_min[a]))
            return fail(RT_ERR_INVALID, "rt_guide_create: empty bounding box");
    if (!(opts->learning_rate > 0)) return fail(RT_ERR_INVALID, "rt_guide_create: learning rate must be positive");
    if (opts->record_capacity > kRecNone - 1)
        return fail(RT_ERR_INVALID, "rt_guide_create: record capacity above 4,194,302");
    RTB_CUDA(cudaSetDevice(ctx->device));
    rt_guide *g = new rt_guide();
    g->ctx = ctx;
    g->opts = *opts;
    g->rec_cap = opts->record_capacity ? opts->record_capacity : kRecNone - 1;
    int s = guide_init_params(g);
    if (s != RT_OK) {
        delete g;
        return s;
    }
    *out = g;
    return RT_OK;
}

int rt_guide_reset(rt_guide *g)
{
    if (!g) return fail(RT_ERR_INVALID, "rt_guide_reset: null guide");
    RTB_CUDA(cudaSetDevice(g->ctx->device));
    return guide_init_params(g);
}

}  // extern "C"

// He-uniform hidden layers, Glorot-uniform output layer, zero biases (seeded PCG32)
static int guide_init_params(rt_guide *g)
{
    std::vector<float> p(kGuideParamCount, 0.f);
    uint64_t state = 0x853c49e6748fea9bull ^ ((uint64_t)g->opts.seed << 1);
    auto next = [&]() {
        const uint64_t old = state;
        state = old * 6364136223846793005ull + 1442695040888963407ull;
        const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u), rot = (uint32_t)(old >> 59u);
        const uint32_t r = (xs >> rot) | (xs << ((32u - rot) & 31u));
        return (float)(r >> 8) * (1.0f / 16777216.0f);
    };
    for (int l = 0; l < kGuideLayers; l++) {
        const int in = guide_in(l), o = guide_out(l);
        const float a = l == kGuideLayers - 1 ? std::sqrt(6.f / (float)(in + o)) : std::sqrt(6.f / (float)in);
        for (int i = 0; i < in * o; i++) p[guide_pw(l) + i] = (2.f * next() - 1.f) * a;
    }
    RTB_CHECK(guide_upload_params(g, p.data()));
    g->trained = false;
    return RT_OK;
}

extern "C" {

int rt_guide_destroy(rt_guide *g)
{
    if (!g) return RT_OK;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    if (g->host_scal) cudaFreeHost(g->host_scal);
    delete g;
    return RT_OK;
}

int rt_guide_param_count(rt_guide *g, uint64_t *n)
{
    if (!g || !n) return fail(RT_ERR_INVALID, "rt_guide_param_count: null argument");
    *n = kGuideParamCount;
    return RT_OK;
}

int rt_guide_params_get(rt_guide *g, float *host, uint64_t n)
{
    if (!g || !host) return fail(RT_ERR_INVALID, "rt_guide_params_get: null argument");
    if (n != (uint64_t)kGuideParamCount) return fail(RT_ERR_INVALID, "rt_guide_params_get: wrong parameter count");
    RTB_CUDA(cudaSetDevice(g->ctx->device));
    RTB_CUDA(cudaMemcpyAsync(host, g->master.ptr, 4ull * n, cudaMemcpyDeviceToHost, g->ctx->stream));
    RTB_CUDA(cudaStreamSynchronize(g->ctx->stream));
    return RT_OK;
}

int rt_guide_params_set(rt_guide *g, const float *host, uint64_t n)
{
    if (!g || !host) return fail(RT_ERR_INVALID, "rt_guide_params_set: null argument");
    if (n != (uint64_t)kGuideParamCount) return fail(RT_ERR_INVALID, "rt_guide_params_set: wrong parameter count");
    for (uint64_t i = 0; i < n; i++)
        if (!std::isfinite(host[i])) return fail(RT_ERR_INVALID, "rt_guide_params_set: non-finite parameter");
    RTB_CUDA(cudaSetDevice(g->ctx->device));
    RTB_CHECK(guide_upload_params(g, host));
    g->trained = true;
    return RT_OK;
}

int rt_guide_steps(rt_guide *g, uint64_t *steps)
{
    if (!g || !steps) return fail(RT_ERR_INVALID, "rt_guide_steps: null argument");
    *steps = g->step;
    return RT_OK;
}

static int guide_eval_common(rt_guide *g, uint64_t B, const char *who)
{
    if (!g) return fail(RT_ERR_INVALID, std::string(who) + ": null guide");
    if (B >= (1ull << 31)) return fail(RT_ERR_INVALID, std::string(who) + ": batch too large");
    RTB_CUDA(cudaSetDevice(g->ctx->device));
    if (!(device_slot(SLOT_SMEM_ATTRS) & SMEM_GUIDE_EVAL)) {
        RTB_CUDA(cudaFuncSetAttribute(k_guide_eval<RawSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem));
        RTB_CUDA(cudaFuncSetAttribute(k_guide_eval<PdfSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem));
        RTB_CUDA(
            cudaFuncSetAttribute(k_guide_eval<SampleSink>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem));
        or_device_slot(SLOT_SMEM_ATTRS, SMEM_GUIDE_EVAL);
    }
    return RT_OK;
}

static unsigned infer_grid(rt_guide *g, uint64_t B)
{
    const uint64_t tiles = (B + kInferRows - 1) / kInferRows;
    return (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((tiles + kInferGroups - 1) / kInferGroups, (uint64_t)std::max(g->ctx->sm_count, 1)));
}

// zeroes the tensor-core wait flag before an evaluation launch
static int guide_eval_begin(rt_guide *g)
{
    RTB_CHECK(g->werr.reserve(16));
    RTB_CUDA(cudaMemsetAsync(g->werr.ptr, 0, 4, g->ctx->stream));
    return RT_OK;
}

// waits for the evaluation and reports a tensor-core wait that ran out
static int guide_eval_end(rt_guide *g, const char *who)
{
    uint32_t werr = 0;
    RTB_CUDA(cudaMemcpyAsync(&werr, g->werr.ptr, 4, cudaMemcpyDeviceToHost, g->ctx->stream));
    RTB_CUDA(cudaStreamSynchronize(g->ctx->stream));
    if (werr) return fail(RT_ERR_TIMEOUT, std::string(who) + ": tensor-core completion wait timed out");
    return RT_OK;
}

int rt_guide_eval(rt_guide *g, const float *queries, uint64_t B, float *out)
{
    RTB_CHECK(guide_eval_common(g, B, "rt_guide_eval"));
    if (B == 0) return RT_OK;
    if (!queries || !out) return fail(RT_ERR_INVALID, "rt_guide_eval: null buffer");
    RTB_CHECK(guide_eval_begin(g));
    k_guide_eval<RawSink><<<infer_grid(g, B), kInferWarps * 32, kInferSmem, g->ctx->stream>>>(
        g->img.as<uint4>(), guide_box(g), (uint32_t)B, QuerySrc{queries}, RawSink{out}, g->werr.as<uint32_t>());
    RTB_CUDA(cudaGetLastError());
    return guide_eval_end(g, "rt_guide_eval");
}

int rt_guide_pdf(rt_guide *g, const float *queries, const float *dirs, const float *bsdf_pdf, uint64_t B, float *out)
{
    RTB_CHECK(guide_eval_common(g, B, "rt_guide_pdf"));
    if (B == 0) return RT_OK;
    if (!queries || !dirs || !bsdf_pdf || !out) return fail(RT_ERR_INVALID, "rt_guide_pdf: null buffer");
    RTB_CHECK(guide_eval_begin(g));
    k_guide_eval<PdfSink><<<infer_grid(g, B), kInferWarps * 32, kInferSmem, g->ctx->stream>>>(
        g->img.as<uint4>(), guide_box(g), (uint32_t)B, QuerySrc{queries}, PdfSink{dirs, bsdf_pdf, out}, g->werr.as<uint32_t>());
    RTB_CUDA(cudaGetLastError());
    return guide_eval_end(g, "rt_guide_pdf");
}

int rt_guide_sample(rt_guide *g, const float *queries, const float *u3, uint64_t B, float *out_dirs, float *out_pdf)
{
    RTB_CHECK(guide_eval_common(g, B, "rt_guide_sample"));
    if (B == 0) return RT_OK;
    if (!queries || !u3 || !out_dirs || !out_pdf) return fail(RT_ERR_INVALID, "rt_guide_sample: null buffer");
    RTB_CHECK(guide_eval_begin(g));
    k_guide_eval<SampleSink><<<infer_grid(g, B), kInferWarps * 32, kInferSmem, g->ctx->stream>>>(
        g->img.as<uint4>(), guide_box(g), (uint32_t)B, QuerySrc{queries}, SampleSink{u3, out_dirs, out_pdf}, g->werr.as<uint32_t>());
    RTB_CUDA(cudaGetLastError());
    return guide_eval_end(g, "rt_guide_sample");
}

int rt_guide_train_step(rt_guide *g, const float *queries, const float *dirs, const float *bsdf_pdf,
                        const float *weights, uint64_t B, int apply, float *grad_host, float *loss_out)
{
    if (!g) return fail(RT_ERR_INVALID, "rt_guide_train_step: null guide");
    if (B && (!queries || !dirs || !bsdf_pdf || !weights))
        return fail(RT_ERR_INVALID, "rt_guide_train_step: null buffer");
    if (B >= (1ull << 31)) return fail(RT_ERR_INVALID, "rt_guide_train_step: batch too large");
    RTB_CUDA(cudaSetDevice(g->ctx->device));
    return guide_train(g, queries, dirs, bsdf_pdf, weights, B, apply, grad_host, loss_out);
}

int rt_render_set_guide(rt_scene *s, rt_guide *g, int train)
{
    if (!s) return fail(RT_ERR_INVALID, "rt_render_set_guide: null scene");
    if (g && g->ctx->device != s->ctx->device) return fail(RT_ERR_INVALID, "rt_render_set_guide: device mismatch");
    s->guide = g;
    s->guide_train = g ? (train != 0) : 0;
    return RT_OK;
}

int rt_guide_record_count(rt_guide *g, uint64_t *records, uint64_t *nonzero)
{
    if (!g) return fail(RT_ERR_INVALID, "rt_guide_record_count: null guide");
    uint32_t c[2] = {0, 0};
    if (g->rcnt.ptr) {
        RTB_CUDA(cudaSetDevice(g->ctx->device));
        RTB_CUDA(cudaMemcpyAsync(c, g->rcnt.ptr, 8, cudaMemcpyDeviceToHost, g->ctx->stream));
        RTB_CUDA(cudaStreamSynchronize(g->ctx->stream));
    }
    if (records) *records = std::min(c[0], g->rec_cap);
    if (nonzero) *nonzero = std::min(c[1], g->rec_cap);
    return RT_OK;
}

int rt_guide_records_get(rt_guide *g, uint64_t first, uint64_t n, float *host)
{
    if (!g || (!host && n)) return fail(RT_ERR_INVALID, "rt_guide_records_get: null argument");
    uint64_t have = 0;
    RTB_CHECK(rt_guide_record_count(g, &have, nullptr));
    if (first + n > have) return fail(RT_ERR_INVALID, "rt_guide_records_get: range beyond the recorded samples");
    if (n == 0) return RT_OK;
    RTB_CUDA(cudaMemcpyAsync(host, g->recs.as<GuideRecord>() + first, sizeof(GuideRecord) * n, cudaMemcpyDeviceToHost,
                             g->ctx->stream));
    RTB_CUDA(cudaStreamSynchronize(g->ctx->stream));
    return RT_OK;
}

int rt_guide_train_records(rt_guide *g, uint32_t steps, uint32_t batch, uint32_t seed, float *loss_out)
{
    if (!g) return fail(RT_ERR_INVALID, "rt_guide_train_records: null guide");
    if (batch == 0 || batch >= (1u << 30)) return fail(RT_ERR_INVALID, "rt_guide_train_records: bad batch size");
    uint64_t nnz = 0;
    RTB_CHECK(rt_guide_record_count(g, nullptr, &nnz));
    if (loss_out) *loss_out = 0.f;
    if (nnz == 0 || steps == 0) return RT_OK;
    cudaStream_t st = g->ctx->stream;
    RTB_CHECK(g->tq.reserve(36ull * batch));
    RTB_CHECK(g->tdir.reserve(12ull * batch));
    RTB_CHECK(g->tpdf.reserve(4ull * batch));
    RTB_CHECK(g->tw.reserve(4ull * batch));
    for (uint32_t k = 0; k < steps; k++) {
        k_guide_gather<<<(batch + 255) / 256, 256, 0, st>>>(
            g->recs.as<GuideRecord>(), g->nz.as<uint32_t>(), (uint32_t)nnz, batch,
            seed * 0x9E3779B9u + (uint32_t)g->step * 0x85EBCA6Bu + k, g->tq.as<float>(), g->tdir.as<float>(),
            g->tpdf.as<float>(), g->tw.as<float>());
        RTB_CUDA(cudaGetLastError());
        RTB_CHECK(guide_train(g, g->tq.as<float>(), g->tdir.as<float>(), g->tpdf.as<float>(), g->tw.as<float>(), batch,
                              1, nullptr, (k + 1 == steps) ? loss_out : nullptr));
    }
    return RT_OK;
}

}  // extern "C"
