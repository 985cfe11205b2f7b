// Film output and comparison: the reference's .hdrbmp accumulation files
// (Film::storeContributionsToFile / loadContributionsFromFile, camera/Film.cu:366-449), its
// computeRMSE (camera/Film.cu:611-632), and its tone mapping to 8-bit images with the BMP and
// PPM writers (Film::toneMaxPixel, writeToBMP, writeToPPM, camera/Film.cu:120-360,
// camera/BMP_Format.cu), for films the renderer accumulates on the device.
#include <cmath>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "rt_internal.h"
#include "tonemap.cuh"

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

// The film pixel as the reference holds it: the sum over `samples` samples, the invalid ones
// replaced by the mean of the valid ones (pathTracing.cu:457-490), as rt_film_store_hdrbmp
// writes it.
__device__ __forceinline__ D3 film_pixel(const float *s, const uint32_t *c, const double *s64, uint64_t i,
                                         double samples)
{
    D3 p = s64 ? D3{s64[3 * i], s64[3 * i + 1], s64[3 * i + 2]} : D3{s[3 * i], s[3 * i + 1], s[3 * i + 2]};
    if (c) {
        const double k = c[i] ? td_div(samples, (double)c[i]) : 0.0;
        p = p * k;
    }
    return p;
}

constexpr int kTmBlocks = 592, kTmThreads = 256;

// Film::getMaxChannel / getMaxLuminance (Film.cu:120-153) before their division by the
// sample count: per-block maxima of the channels and of Spectrum::brightness, from 0.
__global__ void __launch_bounds__(kTmThreads) k_tm_max(const float *s, const uint32_t *c, const double *s64,
                                                       uint64_t npix, double samples, double *partial)
{
    __shared__ double red[2][kTmThreads];
    double mc = 0.0, ml = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)kTmThreads + threadIdx.x; i < npix; i += (uint64_t)gridDim.x * kTmThreads) {
        const D3 p = film_pixel(s, c, s64, i, samples);
        if (p.r > mc) mc = p.r;
        if (p.g > mc) mc = p.g;
        if (p.b > mc) mc = p.b;
        const double l = tm_brightness(p);
        if (l > ml) ml = l;
    }
    red[0][threadIdx.x] = mc;
    red[1][threadIdx.x] = ml;
    __syncthreads();
    for (int o = kTmThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            if (red[0][threadIdx.x + o] > red[0][threadIdx.x]) red[0][threadIdx.x] = red[0][threadIdx.x + o];
            if (red[1][threadIdx.x + o] > red[1][threadIdx.x]) red[1][threadIdx.x] = red[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x < 2) partial[2 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

// the film maxima over the blocks' partial maxima, divided by the sample count
__global__ void k_tm_final(const double *partial, int nblocks, double samples, double *mm)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mc = 0.0, ml = 0.0;
    for (int b = 0; b < nblocks; b++) {
        if (partial[2 * b] > mc) mc = partial[2 * b];
        if (partial[2 * b + 1] > ml) ml = partial[2 * b + 1];
    }
    mm[0] = td_div(mc, samples);
    mm[1] = td_div(ml, samples);
}

__global__ void __launch_bounds__(kTmThreads) k_tm_map(const float *s, const uint32_t *c, const double *s64,
                                                       uint64_t npix, double samples, uint32_t mode,
                                                       const double *mm, uint8_t *rgb)
{
    const uint64_t i = blockIdx.x * (uint64_t)kTmThreads + threadIdx.x;
    if (i >= npix) return;
    const D3 q = tonemap_pixel(film_pixel(s, c, s64, i, samples), samples, mm[0], mm[1], mode);
    rgb[3 * i] = tm_byte(q.r);
    rgb[3 * i + 1] = tm_byte(q.g);
    rgb[3 * i + 2] = tm_byte(q.b);
}

template <class T>
void put(std::ofstream &f, T v)  // little-endian field, as BitmapImage writes it on x86
{
    f.write(reinterpret_cast<const char *>(&v), sizeof(T));
}

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

int rt_film_tonemap(const float *sum_rgb, const uint32_t *count, const double *sum64, uint64_t npix, uint64_t samples,
                    uint32_t mode, uint8_t *rgb8)
{
    if ((!sum_rgb && !sum64) || !rgb8) return fail(RT_ERR_INVALID, "rt_film_tonemap: null argument");
    if (npix == 0 || samples == 0) return fail(RT_ERR_INVALID, "rt_film_tonemap: empty film");
    if (mode > RT_TONEMAP_GAMMA_CLAMP) return fail(RT_ERR_INVALID, "rt_film_tonemap: unknown mode");
    double *scratch = nullptr;  // per-block maxima, then the two film maxima
    RTB_CUDA(cudaMalloc(&scratch, sizeof(double) * (2 * kTmBlocks + 2)));
    const double ns = (double)samples;
    k_tm_max<<<kTmBlocks, kTmThreads>>>(sum_rgb, count, sum64, npix, ns, scratch);
    k_tm_final<<<1, 32>>>(scratch, kTmBlocks, ns, scratch + 2 * kTmBlocks);
    k_tm_map<<<(unsigned)((npix + kTmThreads - 1) / kTmThreads), kTmThreads>>>(sum_rgb, count, sum64, npix, ns, mode,
                                                                              scratch + 2 * kTmBlocks, rgb8);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(scratch);
    if (e != cudaSuccess) return cuda_status(e, "rt_film_tonemap");
    return RT_OK;
}

int rt_image_write_bmp(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height)
{
    if (!path || !rgb8 || !width || !height) return fail(RT_ERR_INVALID, "rt_image_write_bmp: bad argument");
    std::ofstream f(path, std::ios::binary);
    if (!f.is_open()) return fail(RT_ERR_INVALID, std::string("rt_image_write_bmp: cannot open ") + path);
    // BitmapImage (camera/BMP_Format.cu): 14-byte file header, 40-byte info header whose image
    // size field is (width + 4 - width % 4) * height, then bottom-up rows of BGR bytes, each
    // padded with zero bytes to a multiple of 4
    const uint32_t image_size = (width + 4 - (width % 4)) * height;
    f.write("BM", 2);
    put<uint32_t>(f, 14 + 40 + image_size);
    put<uint16_t>(f, 0);
    put<uint16_t>(f, 0);
    put<uint32_t>(f, 14 + 40);
    put<uint32_t>(f, 40);
    put<int32_t>(f, (int32_t)width);
    put<int32_t>(f, (int32_t)height);
    put<uint16_t>(f, 1);
    put<uint16_t>(f, 24);
    put<uint32_t>(f, 0);
    put<uint32_t>(f, image_size);
    put<uint32_t>(f, 3780);
    put<uint32_t>(f, 3780);
    put<uint32_t>(f, 0);
    put<uint32_t>(f, 0);
    std::vector<char> row(((3 * (size_t)width + 3) / 4) * 4, 0);
    for (uint32_t i = 0; i < height; i++) {
        const uint8_t *src = rgb8 + 3 * (size_t)width * (height - 1 - i);  // film rows top to bottom
        for (uint32_t j = 0; j < width; j++) {
            row[3 * j] = (char)src[3 * j + 2];
            row[3 * j + 1] = (char)src[3 * j + 1];
            row[3 * j + 2] = (char)src[3 * j];
        }
        f.write(row.data(), (std::streamsize)row.size());
    }
    f.close();
    if (!f) return fail(RT_ERR_INVALID, "rt_image_write_bmp: write failed");
    return RT_OK;
}

int rt_image_write_ppm(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height)
{
    if (!path || !rgb8 || !width || !height) return fail(RT_ERR_INVALID, "rt_image_write_ppm: bad argument");
    std::ofstream f(path, std::ios::binary);
    if (!f.is_open()) return fail(RT_ERR_INVALID, std::string("rt_image_write_ppm: cannot open ") + path);
    f << "P6\n" << width << " " << height << "\n255\n";  // Film::writeToPPM
    f.write(reinterpret_cast<const char *>(rgb8), (std::streamsize)(3 * (size_t)width * height));
    f.close();
    if (!f) return fail(RT_ERR_INVALID, "rt_image_write_ppm: write failed");
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
