// Learned path guide: device-side pieces shared by the training kernels (guide.cu) and the
// path tracer (render.cu). The reference renderer has no counterpart; this is the estimator's
// importance-sampling proposal, combined with BSDF sampling by one-sample MIS.
//
// Network: 144 encoded inputs -> 4 hidden layers of 64 (ReLU) -> 48 outputs, FP16 weights and
// activations on the 5th-generation tensor cores (tcgen05.mma, FP32 accumulators in TMEM) for
// inference and training, FP32 master weights.
// Input encoding of a shading point (position p, shading normal n, outgoing direction wo):
//   [0, 72)    p normalised to the guide's box (u in [0, 1]), per axis 12 frequency bands:
//              sin, cos(2^(k/2) pi u), k = 0..11 (half-octave steps: the finest band resolves
//              about 1/90 of the box, the scale of the lighting detail, not of the geometry)
//   [72, 104)  theta(wo) / pi, one-blob over 32 bins (Gaussian, sigma = 1/32)
//   [104, 136) phi(wo) / 2pi + 1/2, one-blob over 32 bins
//   [136, 139) n;  [139, 144) zero
// Outputs per lobe j (8 von Mises-Fisher lobes): o[4j] -> theta = pi sigmoid, o[4j+1] -> phi =
// 2 pi sigmoid, o[4j+2] -> kappa = exp(-4 + 12 sigmoid), o[4j+3] -> softmax weight logit;
// o[32] -> alpha = 0.05 + 0.9 sigmoid, the probability of sampling the guide. o[33..47] unused.
#pragma once

#include <cuda_fp16.h>

#include "shading.cuh"

namespace rtb {

constexpr int kGuideIn = 144, kGuideHidden = 64, kGuideOut = 48, kGuideLayers = 5, kGuideLobes = 8;
constexpr int kGuideParamCount = 24880;  // 144*64+64 + 3*(64*64+64) + 64*48+48
constexpr float kGuideAlphaMin = 0.05f, kGuideAlphaSpan = 0.9f;  // alpha in [0.05, 0.95]
constexpr float kGuideLogKappaMin = -4.f, kGuideLogKappaSpan = 12.f;  // log kappa in (-4, 8)
constexpr float kGuideWeightClip = 32.f;    // training weight / batch mean is clipped here
constexpr float kGuideGradClamp = 8192.f;  // per-output gradient clamp
constexpr float kGuideGradScale = 8.f;     // output gradients are stored as fp16(g / scale)

// path-state record link: bits [10, 32) of the flags word
constexpr uint32_t kRecNone = 0x3FFFFFu;
constexpr int kRecShift = 10;

__host__ __device__ constexpr int guide_in(int l) { return l == 0 ? kGuideIn : kGuideHidden; }
__host__ __device__ constexpr int guide_out(int l) { return l == kGuideLayers - 1 ? kGuideOut : kGuideHidden; }
// FP32 master parameters: for each layer W_l (in x out, row-major), then b_l
__host__ __device__ constexpr int guide_pw(int l)
{
    return l == 0 ? 0 : guide_pw(l - 1) + guide_in(l - 1) * guide_out(l - 1) + guide_out(l - 1);
}
__host__ __device__ constexpr int guide_pb(int l) { return guide_pw(l) + guide_in(l) * guide_out(l); }
static_assert(guide_pb(4) + 48 == kGuideParamCount, "parameter count");

// FP16 weight image (the shared-memory copy, loaded with 16-byte copies): W_l transposed,
// out_l rows of stride guide_stride(l) halves (the kernels restage them as core matrices), then
// the FP32 biases (64 per hidden layer, 48 for the output layer).
__host__ __device__ constexpr int guide_stride(int l) { return l == 0 ? 152 : 72; }
__host__ __device__ constexpr int guide_iw(int l)
{
    return l == 0 ? 0 : guide_iw(l - 1) + guide_out(l - 1) * guide_stride(l - 1);
}
constexpr int kGuideImgHalves = 64 * 152 + 3 * 64 * 72 + 48 * 72;
static_assert(guide_iw(4) + 48 * 72 == kGuideImgHalves, "image layout");
constexpr int kGuideImgBias = kGuideImgHalves * 2;  // byte offset of the biases
__host__ __device__ constexpr int guide_ib(int l) { return l * 64; }  // float index of b_l
constexpr int kGuideImgBytes = kGuideImgBias + 4 * (4 * 64 + 48);
static_assert(kGuideImgBias % 16 == 0 && kGuideImgBytes % 16 == 0, "image alignment");

// transposed activations / gradients for the weight-gradient kernel: feature-major planes
__host__ __device__ constexpr int guide_xoff(int l) { return l == 0 ? 0 : kGuideIn + (l - 1) * kGuideHidden; }
__host__ __device__ constexpr int guide_goff(int l) { return l * kGuideHidden; }
constexpr int kGuideXFeatures = kGuideIn + 4 * kGuideHidden;   // 400
constexpr int kGuideGFeatures = 4 * kGuideHidden + kGuideOut;  // 304

// Per queue slot: the decoded mixture at the path's current hit (written by the inference
// kernel, read by shading). alpha = 0 marks a hit that is not guided.
struct GuideParams {
    float4 lobe[kGuideLobes];  // mean direction xyz (world), concentration
    float lam[kGuideLobes];    // lobe weights, sum 1
    float lamn[kGuideLobes];   // lam * vMF normalisation
    float alpha;
    float pad[3];
};
static_assert(sizeof(GuideParams) == 208, "GuideParams layout");

// One training sample: a guided vertex of a traced path.
struct GuideRecord {
    float4 a;  // position xyz, normal x
    float4 b;  // normal yz, wo xy
    float4 c;  // wo z, sampled direction wi xyz
    float4 d;  // BSDF sampling pdf of wi, path throughput before the vertex rgb
    float4 e;  // radiance arriving after the vertex rgb (its suffix sum once the path retired),
               // previous record of the path (uint bits, kRecNone: none)
};
static_assert(sizeof(GuideRecord) == 80, "GuideRecord layout");

struct GuideBox {
    float3 lo, inv_ext;
};
}  // namespace rtb
struct rt_guide;
namespace rtb {
GuideBox guide_box(const rt_guide *g);  // position encoding domain of a guide

// ------------------------------------------------------------------ encoding

// one-blob Gaussian: |d| > 6 bins gives exp(-18) < 2^-25, which rounds to FP16 zero, so the
// fast exponential's flush of tiny results changes no encoded value
__device__ __forceinline__ float guide_blob(float x, int i)
{
    const float d = x * 32.f - ((float)i + 0.5f);
    return __expf(-0.5f * d * d);
}

// part 0: position bands (half2 0..35); part 1: direction blobs, normal, zero pad (36..71)
__device__ __forceinline__ void guide_encode(int part, const float *q, const GuideBox &bx, __half2 *row)
{
    if (part == 0) {
        const float u[3] = {fminf(fmaxf((q[0] - bx.lo.x) * bx.inv_ext.x, 0.f), 1.f),
                            fminf(fmaxf((q[1] - bx.lo.y) * bx.inv_ext.y, 0.f), 1.f),
                            fminf(fmaxf((q[2] - bx.lo.z) * bx.inv_ext.z, 0.f), 1.f)};
        // band k + 2 doubles the angle of band k: sin 2x = 2 sin x cos x, cos 2x = cos^2 x -
        // sin^2 x, from sincospi(u) and sincospi(sqrt(2) u); five doublings grow the absolute
        // error to ~2e-6, far below the FP16 step of the encoded value
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float s0, c0, s1, c1;
            sincospif(u[a], &s0, &c0);
            sincospif(u[a] * 1.41421356f, &s1, &c1);
#pragma unroll
            for (int k = 0; k < 12; k += 2) {
                row[a * 12 + k] = __floats2half2_rn(s0, c0);
                row[a * 12 + k + 1] = __floats2half2_rn(s1, c1);
                const float s0n = 2.f * s0 * c0, c0n = fmaf(c0, c0, -s0 * s0);
                const float s1n = 2.f * s1 * c1, c1n = fmaf(c1, c1, -s1 * s1);
                s0 = s0n, c0 = c0n, s1 = s1n, c1 = c1n;
            }
        }
    } else {
        const float th = acosf(fminf(fmaxf(q[8], -1.f), 1.f)) * (1.f / 3.14159265358979f);
        const float ph = atan2f(q[7], q[6]) * (1.f / 6.28318530717959f) + 0.5f;
#pragma unroll
        for (int i = 0; i < 16; i++) row[36 + i] = __floats2half2_rn(guide_blob(th, 2 * i), guide_blob(th, 2 * i + 1));
#pragma unroll
        for (int i = 0; i < 16; i++) row[52 + i] = __floats2half2_rn(guide_blob(ph, 2 * i), guide_blob(ph, 2 * i + 1));
        row[68] = __floats2half2_rn(q[3], q[4]);
        row[69] = __floats2half2_rn(q[5], 0.f);
        row[70] = __floats2half2_rn(0.f, 0.f);
        row[71] = __floats2half2_rn(0.f, 0.f);
    }
}

// ------------------------------------------------------------------ vMF mixture

__device__ __forceinline__ float guide_sigmoid(float x) { return 1.f / (1.f + expf(-x)); }
// the decode's sigmoid: the mixture is decoded once per hit and both the sampling and the
// density use the decoded lobes, so a few ulp here only move the network's function
__device__ __forceinline__ float guide_sigmoid_fast(float x) { return __fdividef(1.f, 1.f + __expf(-x)); }

// kappa / (2 pi (1 - exp(-2 kappa))): the vMF density is norm * exp(kappa (mu.w - 1))
__device__ __forceinline__ float vmf_norm(float k) { return k / (6.28318530717959f * (-expm1f(-2.f * k))); }

__device__ __forceinline__ void guide_decode(const float *o, GuideParams &P)
{
    float lmax = o[3];
#pragma unroll
    for (int j = 1; j < kGuideLobes; j++) lmax = fmaxf(lmax, o[4 * j + 3]);
    float e[kGuideLobes], se = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        e[j] = __expf(o[4 * j + 3] - lmax);
        se += e[j];
    }
    const float inv = 1.f / se;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float th = 3.14159265358979f * guide_sigmoid_fast(o[4 * j]);
        const float ph = 6.28318530717959f * guide_sigmoid_fast(o[4 * j + 1]);
        const float k = __expf(kGuideLogKappaMin + kGuideLogKappaSpan * guide_sigmoid_fast(o[4 * j + 2]));
        float st, ct, sp, cp;
        sincosf(th, &st, &ct);
        sincosf(ph, &sp, &cp);
        P.lobe[j] = make_float4(st * cp, st * sp, ct, k);
        P.lam[j] = e[j] * inv;
        P.lamn[j] = P.lam[j] * vmf_norm(k);
    }
    P.alpha = kGuideAlphaMin + kGuideAlphaSpan * guide_sigmoid_fast(o[32]);
}

// mixture density of the vMF lobes at world direction w (unit)
__device__ __forceinline__ float guide_pdf(const GuideParams &P, V3 w)
{
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float4 l = P.lobe[j];
        s += P.lamn[j] * expf(l.w * (l.x * w.x + l.y * w.y + l.z * w.z - 1.f));
    }
    return s;
}

// vMF mixture sample: lobe by u0, direction by the inversion of Jakob (2012), "Numerically
// stable sampling of the von Mises Fisher distribution on S2".
__device__ __forceinline__ V3 guide_sample(const GuideParams &P, float u0, float u1, float u2)
{
    int j = 0;
    float c = P.lam[0];
    while (j < kGuideLobes - 1 && u0 >= c) c += P.lam[++j];
    const float4 l = P.lobe[j];
    const float xi = 1.f - u1;  // (0, 1]
    float w = 1.f + logf(xi + (1.f - xi) * expf(-2.f * l.w)) / l.w;
    w = fminf(fmaxf(w, -1.f), 1.f);
    const float s = sqrtf(fmaxf(0.f, 1.f - w * w));
    float sp, cp;
    sincospif(2.f * u2, &sp, &cp);
    V3 mu = v3(l.x, l.y, l.z), t, b;
    onb(mu, t, b);
    return normalize(t * (s * cp) + b * (s * sp) + mu * w);
}

// Training loss of one sample and its gradient with respect to the raw outputs. The lobes are
// fitted to the sampled integrand on their own (KL divergence), and the selection probability
// alpha minimises the estimator's second moment with the lobes held fixed, so a guide that
// starts out worse than the BSDF still learns and alpha follows what the guide is worth:
//   loss = -wt * log V(wi) + wt^2 * qc / q,   q = alpha * Vc + (1 - alpha) * pdf_bsdf,
// V the vMF mixture; Vc and qc are V and q held constant (the second term trains alpha only;
// its value is wt^2). log V is a log-sum-exp over the lobes, so samples far from every lobe
// keep a gradient.
// dout[0..47] receives the gradient (clamped to +-kGuideGradClamp; 0 for the unused outputs).
__device__ __forceinline__ float guide_loss_grad(const float *o, V3 wi, float pdfb, float wt, float *dout)
{
    float lmax = o[3];
#pragma unroll
    for (int j = 1; j < kGuideLobes; j++) lmax = fmaxf(lmax, o[4 * j + 3]);
    float se = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) se += expf(o[4 * j + 3] - lmax);
    const float lse_l = lmax + logf(se);
    float ls[kGuideLobes], kap[kGuideLobes], cj[kGuideLobes];
    float lsmax = -INFINITY;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float th = 3.14159265358979f * guide_sigmoid(o[4 * j]);
        const float ph = 6.28318530717959f * guide_sigmoid(o[4 * j + 1]);
        const float lk = kGuideLogKappaMin + kGuideLogKappaSpan * guide_sigmoid(o[4 * j + 2]);
        kap[j] = expf(lk);
        float st, ct, sp, cp;
        sincosf(th, &st, &ct);
        sincosf(ph, &sp, &cp);
        cj[j] = st * cp * wi.x + st * sp * wi.y + ct * wi.z;
        // log(lam_j * norm_j * exp(kappa_j (c_j - 1)))
        ls[j] = (o[4 * j + 3] - lse_l) + lk - 1.83787706640935f - logf(-expm1f(-2.f * kap[j])) +
                kap[j] * (cj[j] - 1.f);
        lsmax = fmaxf(lsmax, ls[j]);
    }
    float sv = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) sv += expf(ls[j] - lsmax);
    const float logV = lsmax + logf(sv);
    const float V = expf(logV);
    const float sa = guide_sigmoid(o[32]);
    const float alpha = kGuideAlphaMin + kGuideAlphaSpan * sa;
    const float q = fmaxf(alpha * V + (1.f - alpha) * pdfb, 1e-30f);
    auto clampg = [](float g) { return fminf(fmaxf(g, -kGuideGradClamp), kGuideGradClamp); };
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float sth = guide_sigmoid(o[4 * j]), sph = guide_sigmoid(o[4 * j + 1]);
        const float th = 3.14159265358979f * sth, ph = 6.28318530717959f * sph;
        float st, ct, sp, cp;
        sincosf(th, &st, &ct);
        sincosf(ph, &sp, &cp);
        const float r = expf(ls[j] - logV);  // share of lobe j in V(wi)
        const float k = kap[j];
        const float lam = expf(o[4 * j + 3] - lse_l);
        const float dth = r * k * (ct * cp * wi.x + ct * sp * wi.y - st * wi.z) * 3.14159265358979f * sth * (1.f - sth);
        const float dph = r * k * (-st * sp * wi.x + st * cp * wi.y) * 6.28318530717959f * sph * (1.f - sph);
        const float sk = guide_sigmoid(o[4 * j + 2]);
        const float dk = r * (1.f - 2.f * k / expm1f(2.f * k) + k * (cj[j] - 1.f)) * kGuideLogKappaSpan * sk * (1.f - sk);
        dout[4 * j + 0] = clampg(-wt * dth);
        dout[4 * j + 1] = clampg(-wt * dph);
        dout[4 * j + 2] = clampg(-wt * dk);
        dout[4 * j + 3] = clampg(-wt * (r - lam));
    }
    dout[32] = clampg(-wt * wt * (V - pdfb) / q * kGuideAlphaSpan * sa * (1.f - sa));
#pragma unroll
    for (int i = 33; i < kGuideOut; i++) dout[i] = 0.f;
    return -wt * logV + wt * wt;
}

// ------------------------------------------------------------------ tcgen05 (UMMA) primitives

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major FP16 operand without swizzle. The operand is a
// grid of core matrices of 8 rows x 16 bytes (rows 16 bytes apart); `lbo` is the byte distance
// between the two core matrices of one K = 16 step, `sbo` between consecutive groups of 8
// rows. Fields: start address >> 4 in bits [0, 14), lbo >> 4 in [16, 30), sbo >> 4 in
// [32, 46), descriptor version 1 (sm_100) in [46, 48), base offset 0, layout 0 (no swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16: A and B FP16, both K-major, FP32
// accumulator (bits [4, 6) = 1), N >> 3 in bits [17, 23), M >> 4 in bits [24, 29).
__host__ __device__ constexpr uint32_t umma_idesc_f16(int m, int n)
{
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, one M x N x 16 step, issued by one thread
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// arrive on the mbarrier once every tcgen05.mma this thread issued has completed
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n\tfence.mbarrier_init.release.cluster;" ::"r"(smem_u32(bar)),
                 "r"(count)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// waits for the phase of `parity` to complete, polling at most `limit` times; false: gave up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core's (async proxy) reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation: executed by one whole warp; the column base is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n\t"
        "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::"r"(smem_u32(slot)),
        "r"(ncols)
        : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (the warp reads lanes 32 (warp % 4)
// + 0..31); the wait is inside the same statement, so the values are complete on return
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];\n\ttcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------------ batched inference

// Tiles of 128 rows run through the network on the tensor cores: per layer, tcgen05.mma
// (M = 128, FP16 operands from shared memory, FP32 accumulator in 64 TMEM columns) issued by
// one thread, then the 128 threads of the tile read their own row back from TMEM for bias,
// ReLU and the FP16 store of the next layer's operand. A CTA holds one copy of the weights
// and kInferGroups independent 128-thread groups, each with its own activation tile, TMEM
// columns, mbarrier and named barrier, so 16 warps per SM hide each other's latency.
// Operands are K-major without swizzle, in core matrices of 8 rows x 8 halves: row r, halves
// [8c, 8c + 8) of an operand with KC chunks per row sit at byte (r / 8) * KC * 128 + c * 128 +
// (r % 8) * 16.
constexpr int kInferRows = 128;
constexpr int kInferGroups = 4;
constexpr int kInferWarps = 4 * kInferGroups;
// byte offset of layer l's weight operand (W_l^T: guide_out(l) rows of guide_in(l) halves)
__host__ __device__ constexpr int tc_w(int l) { return l == 0 ? 0 : tc_w(l - 1) + guide_out(l - 1) * guide_in(l - 1) * 2; }
constexpr int kTcBias = tc_w(kGuideLayers);                                 // 304 FP32 biases
constexpr int kTcA = 50432;                                                 // activation tiles
constexpr int kTcATile = kInferRows * kGuideIn * 2;                         // 128 x 144 halves
constexpr int kTcBar = kTcA + kInferGroups * kTcATile;                      // mbarriers, TMEM base
constexpr int kInferSmem = kTcBar + 8 * kInferGroups + 16;
constexpr int kTmemColsPerGroup = 64;
constexpr int kTmemCols = kTmemColsPerGroup * kInferGroups;  // a power of 2 in [32, 512]
constexpr uint32_t kUmmaWaitPolls = 1u << 22;
static_assert(tc_w(1) == 18432 && tc_w(4) == 43008 && kTcBias == 49152, "operand sizes");
static_assert(kTcBias + 4 * (4 * 64 + 48) <= kTcA && kTcA % 128 == 0 && kTcBar % 8 == 0, "shared layout");
static_assert(kInferSmem <= 227 * 1024, "shared memory per CTA");
static_assert(kTmemCols == 256, "TMEM allocation");

// byte offset of row r, chunk c (8 halves) in an operand of kc chunks per row
__host__ __device__ constexpr uint32_t tc_chunk(uint32_t r, uint32_t c, uint32_t kc)
{
    return (r >> 3) * kc * 128u + c * 128u + (r & 7u) * 16u;
}

__device__ __forceinline__ uint32_t relu_half2(float a, float b)
{
    const __half2 h = __hmax2(__floats2half2_rn(a, b), __float2half2_rn(0.f));
    return *reinterpret_cast<const uint32_t *>(&h);
}

// barrier of the 128 threads of a group (named barrier `id`); returns whether any of them
// passed `v`
__device__ __forceinline__ bool group_sync_or(uint32_t id, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, %2, 128, q;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}

// Forward pass over rows [0, n): src(row, q) fills the 9-float query and says whether the row
// is guided; sink(row, valid, out) receives the 48 raw outputs (biases added; meaningless
// where valid is false). Persistent CTAs
// of kInferWarps warps and kInferSmem bytes of dynamic shared memory, one per SM; the weight
// image is staged once per CTA. A tensor-core wait that runs out of polls sets *werr
// (nullable) and ends the group; the CTA frees its TMEM on exit.
template <class Src, class Sink>
__device__ __forceinline__ void guide_infer_rows(const uint4 *img, const GuideBox &box, uint32_t n, Src &src,
                                                 Sink &sink, uint32_t *werr)
{
    extern __shared__ __align__(128) unsigned char guide_smem[];
    unsigned char *sm = guide_smem;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int grp = tid >> 7, gt = tid & 127;  // group, thread within the group
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kTcBar) + grp;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kTcBar + 8 * kInferGroups);
    // weights: image rows (W_l^T, stride guide_stride(l) halves) to core-matrix chunks
    const unsigned char *ib = reinterpret_cast<const unsigned char *>(img);
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
    if (gt == 0) mbar_init(bar, 1);
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, kTmemCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot + (uint32_t)(kTmemColsPerGroup * grp);  // this group's columns
    const uint32_t tlane = tmem + ((uint32_t)(32 * (warp & 3)) << 16);    // this warp's 32 lanes
    const uint32_t bar_id = 1u + (uint32_t)grp;                           // 0 is __syncthreads
    const float *bias = reinterpret_cast<const float *>(sm + kTcBias);
    unsigned char *A = sm + kTcA + grp * kTcATile;
    uint32_t phase = 0;
    bool failed = false;
    const uint32_t stride = gridDim.x * kInferGroups;
    for (uint32_t tile = blockIdx.x * kInferGroups + grp; !failed && (uint64_t)tile * kInferRows < n; tile += stride) {
        const uint32_t row = tile * kInferRows + gt;
        // rows that are not guided keep whatever their operand row holds: a row of the
        // product depends on its own operand row only, and their outputs are not used
        float q[9];
        const bool valid = row < n && src(row, q);
        if (valid) {
            __half2 e[72];
            guide_encode(0, q, box, e);
            guide_encode(1, q, box, e);
#pragma unroll
            for (int c = 0; c < kGuideIn / 8; c++)
                *reinterpret_cast<uint4 *>(A + tc_chunk(gt, c, kGuideIn / 8)) =
                    *reinterpret_cast<const uint4 *>(&e[4 * c]);
        }
        fence_async_smem();
        tc_fence_before();
        if (!group_sync_or(bar_id, valid)) {  // no guided row in the tile: no network pass
            if (row < n) sink(row, false, q);
            continue;
        }
#pragma unroll 1
        for (int l = 0; l < kGuideLayers && !failed; l++) {
            const int kc = guide_in(l) / 8;
            if (gt == 0) {
                tc_fence_after();
                const uint32_t idesc = umma_idesc_f16(kInferRows, guide_out(l));
                const uint32_t a0 = smem_u32(A), b0 = smem_u32(sm + tc_w(l));
                for (int s = 0; s < kc / 2; s++)
                    umma_f16(tmem, umma_desc(a0 + 256u * s, 128u, 128u * kc), umma_desc(b0 + 256u * s, 128u, 128u * kc),
                             idesc, s > 0 ? 1u : 0u);
                umma_commit(bar);
            }
            // warp-uniform, as the tcgen05.ld below is .sync.aligned
            const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar, phase, kUmmaWaitPolls));
            phase ^= 1u;
            tc_fence_after();
            if (ok && l < kGuideLayers - 1) {
                const float *b = bias + guide_ib(l);
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    float v[16];
                    tmem_ld16(tlane + 16u * h, v);
                    uint32_t w[8];
#pragma unroll
                    for (int j = 0; j < 8; j++)  // ReLU after rounding: the same FP16 value
                        w[j] = relu_half2(v[2 * j] + b[16 * h + 2 * j], v[2 * j + 1] + b[16 * h + 2 * j + 1]);
                    *reinterpret_cast<uint4 *>(A + tc_chunk(gt, 2 * h, 8)) = make_uint4(w[0], w[1], w[2], w[3]);
                    *reinterpret_cast<uint4 *>(A + tc_chunk(gt, 2 * h + 1, 8)) = make_uint4(w[4], w[5], w[6], w[7]);
                }
                fence_async_smem();
            } else if (ok) {
                float o[kGuideOut];
                const float *b = bias + guide_ib(l);
#pragma unroll
                for (int h = 0; h < kGuideOut / 16; h++) tmem_ld16(tlane + 16u * h, o + 16 * h);
#pragma unroll
                for (int j = 0; j < kGuideOut; j++) o[j] += b[j];
                if (row < n) sink(row, valid, o);
            }
            tc_fence_before();
            failed = group_sync_or(bar_id, !ok);
        }
    }
    if (failed) {
        if (gt == 0 && werr) atomicExch(werr, 1u);
        mbar_wait_bounded(bar, phase ^ 1u, kUmmaWaitPolls);  // the commit that timed out, if it ever completes
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        __syncwarp();
        tmem_dealloc(*tslot, kTmemCols);
    }
}

}  // namespace rtb
