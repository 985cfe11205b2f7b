// Film output and comparison: the reference's .hdrbmp accumulation files
// (Film::storeContributionsToFile / loadContributionsFromFile, camera/Film.cu:366-449) and its
// computeRMSE (camera/Film.cu:611-632), for films the renderer accumulates on the device.
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "rt_internal.h"

namespace rtb {
namespace {

// per-block partial sums of |mean_a - mean_b|^2 (double), mean = sum / count
__global__ void k_film_sqdiff(const float *sa, const uint32_t *ca, const double *sa64, const float *sb,
                              const uint32_t *cb, const double *sb64, uint64_t npix, double *partial)
{
    __shared__ double red[256 / 32];
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npix; i += (uint64_t)gridDim.x * blockDim.x) {
        const double na = ca[i] ? (double)ca[i] : 1.0, nb = cb[i] ? (double)cb[i] : 1.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double a = (sa64 ? sa64[3 * i + c] : (double)sa[3 * i + c]) / na;
            const double b = (sb64 ? sb64[3 * i + c] : (double)sb[3 * i + c]) / nb;
            acc += (a - b) * (a - b);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) t += red[w];
        partial[blockIdx.x] = t;
    }
}

constexpr int kRmseBlocks = 592;

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

int rt_film_rmse(const float *sum_a, const uint32_t *count_a, const double *sum64_a, const float *sum_b,
                 const uint32_t *count_b, const double *sum64_b, uint64_t npix, double *rmse)
{
    if (!rmse || !count_a || !count_b || (!sum_a && !sum64_a) || (!sum_b && !sum64_b))
        return fail(RT_ERR_INVALID, "rt_film_rmse: null argument");
    if (npix == 0) return fail(RT_ERR_INVALID, "rt_film_rmse: empty film");
    double *partial = nullptr;
    RTB_CUDA(cudaMalloc(&partial, sizeof(double) * kRmseBlocks));
    k_film_sqdiff<<<kRmseBlocks, 256>>>(sum_a, count_a, sum64_a, sum_b, count_b, sum64_b, npix, partial);
    std::vector<double> h(kRmseBlocks);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), partial, sizeof(double) * kRmseBlocks, cudaMemcpyDeviceToHost);
    cudaFree(partial);
    if (e != cudaSuccess) return cuda_status(e, "rt_film_rmse");
    double t = 0.0;
    for (double v : h) t += v;
    *rmse = std::sqrt(t / (double)npix);
    return RT_OK;
}

int rt_film_store_hdrbmp(const char *path, uint32_t width, uint32_t height, const float *sum_rgb, const uint32_t *count,
                         const double *sum64, uint64_t samples)
{
    if (!path || !count || (!sum_rgb && !sum64)) return fail(RT_ERR_INVALID, "rt_film_store_hdrbmp: null argument");
    const uint64_t npix = (uint64_t)width * height;
    if (npix == 0 || samples == 0) return fail(RT_ERR_INVALID, "rt_film_store_hdrbmp: empty film");
    std::vector<double> s(3 * npix);
    std::vector<uint32_t> c(npix);
    cudaError_t e;
    if (sum64) {
        e = cudaMemcpy(s.data(), sum64, 24 * npix, cudaMemcpyDeviceToHost);
    } else {
        std::vector<float> f(3 * npix);
        e = cudaMemcpy(f.data(), sum_rgb, 12 * npix, cudaMemcpyDeviceToHost);
        for (uint64_t i = 0; i < 3 * npix; i++) s[i] = f[i];
    }
    if (e == cudaSuccess) e = cudaMemcpy(c.data(), count, 4 * npix, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "rt_film_store_hdrbmp");
    std::ofstream file(std::string(path) + ".hdrbmp", std::ios::binary);
    if (!file.is_open()) return fail(RT_ERR_INVALID, std::string("rt_film_store_hdrbmp: cannot open ") + path);
    // header and numbers as the reference writes them (default stream formatting)
    file << "P6\n" << width << " " << height << "F\n" << (long long)samples << "\n";
    for (uint64_t i = 0; i < npix; i++) {
        // the per-pixel sum over `samples` samples, invalid samples replaced by the mean
        // of the valid ones (pathTracing.cu:457-490)
        const double k = c[i] ? (double)samples / c[i] : 0.0;
        file << s[3 * i] * k << " " << s[3 * i + 1] * k << " " << s[3 * i + 2] * k << " ";
    }
    file.close();
    if (!file) return fail(RT_ERR_INVALID, "rt_film_store_hdrbmp: write failed");
    return RT_OK;
}

int rt_film_load_hdrbmp(const char *path, uint32_t width, uint32_t height, double *sum_rgb_host, uint64_t *samples)
{
    if (!path || !sum_rgb_host || !samples) return fail(RT_ERR_INVALID, "rt_film_load_hdrbmp: null argument");
    std::ifstream file(std::string(path) + ".hdrbmp", std::ios::binary);
    if (!file.is_open()) return fail(RT_ERR_INVALID, std::string("rt_film_load_hdrbmp: cannot open ") + path);
    std::string header;
    int w = 0, h = 0;
    char type = 0;
    long long n = 0;
    file >> header >> w >> h >> type >> n;
    if (!file || header != "P6") return fail(RT_ERR_INVALID, "rt_film_load_hdrbmp: not an accumulation file");
    if ((uint32_t)w != width || (uint32_t)h != height)
        return fail(RT_ERR_INVALID, "rt_film_load_hdrbmp: resolution differs from the film's");
    const uint64_t npix = (uint64_t)width * height;
    for (uint64_t i = 0; i < 3 * npix; i++) file >> sum_rgb_host[i];
    if (!file) return fail(RT_ERR_INVALID, "rt_film_load_hdrbmp: truncated file");
    *samples = (uint64_t)n;
    return RT_OK;
}

}  // extern "C"
