// Evaluation and sampling of a material's BSDF on the device for given directions in the
// shading frame (normal +z): the code the renderer runs at every path vertex, exposed for
// tools that tabulate or check a material (Material::lightReflected / pdf / sampleDirection,
// materials/*.cu).
#include "rt_internal.h"
#include "surface.cuh"

namespace rtb {
namespace {

constexpr int kMB = 128;

__global__ void k_material_eval(rt_material m, const float *__restrict__ wo, const float *__restrict__ wi, uint64_t n,
                                float *__restrict__ f, float *__restrict__ pdf)
{
    const uint64_t i = blockIdx.x * (uint64_t)kMB + threadIdx.x;
    if (i >= n) return;
    const Bsdf b = load_bsdf(m);
    float p = 0.f;
    const V3 v = bsdf_eval(b, v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), p);
    f[3 * i] = v.x;
    f[3 * i + 1] = v.y;
    f[3 * i + 2] = v.z;
    if (pdf) pdf[i] = p;
}

__global__ void k_material_sample(rt_material m, const float *__restrict__ wo, uint64_t n, uint32_t seed, int compat,
                                  float *__restrict__ wi, float *__restrict__ value, float *__restrict__ pdf,
                                  uint8_t *__restrict__ delta)
{
    const uint64_t i = blockIdx.x * (uint64_t)kMB + threadIdx.x;
    if (i >= n) return;
    const Bsdf b = load_bsdf(m);
    Pcg r = pcg_init((uint32_t)i, (uint32_t)(i >> 32), seed);
    V3 w;
    float p = 0.f;
    bool d = false;
    const V3 v = bsdf_sample(b, v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), r, compat != 0, w, p, d);
    wi[3 * i] = w.x;
    wi[3 * i + 1] = w.y;
    wi[3 * i + 2] = w.z;
    value[3 * i] = v.x;
    value[3 * i + 1] = v.y;
    value[3 * i + 2] = v.z;
    if (pdf) pdf[i] = p;
    if (delta) delta[i] = d ? 1 : 0;
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

int rt_material_eval(const rt_material *m, const float *wo, const float *wi, uint64_t n, float *f, float *pdf)
{
    if (!m || (n && (!wo || !wi || !f))) return fail(RT_ERR_INVALID, "rt_material_eval: null argument");
    if (n == 0) return RT_OK;
    k_material_eval<<<(unsigned)((n + kMB - 1) / kMB), kMB>>>(*m, wo, wi, n, f, pdf);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaDeviceSynchronize());
    return RT_OK;
}

int rt_material_sample(const rt_material *m, const float *wo, uint64_t n, uint32_t seed, uint32_t flags, float *wi,
                       float *value, float *pdf, uint8_t *delta)
{
    if (!m || (n && (!wo || !wi || !value))) return fail(RT_ERR_INVALID, "rt_material_sample: null argument");
    if (n == 0) return RT_OK;
    k_material_sample<<<(unsigned)((n + kMB - 1) / kMB), kMB>>>(*m, wo, n, seed, (flags & RT_RENDER_COMPAT) ? 1 : 0, wi,
                                                               value, pdf, delta);
    RTB_CUDA(cudaGetLastError());
    RTB_CUDA(cudaDeviceSynchronize());
    return RT_OK;
}

}  // extern "C"
