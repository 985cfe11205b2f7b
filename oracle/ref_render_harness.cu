// Test infrastructure only: runs the reference renderer's OWN integrator
// (PathTracerIntegrator::render, integration/PathTracerIntegrator.cu:140-210, with its bounce
// loop computeSamples, pathTracing.cu:284-414) on a scene the reference can render without
// its GPU BVH: Plane shapes (shapes/Plane.cu), Lambertian materials and the camera and point
// lights read by its own .obejota loader (cuda_libraries/FileImporting.cu:466). The
// reference's compile-time configuration (types.h:41-87) is set for the test image below.
//
// Used by the statistical image-parity test only; the product never links it.
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/sequence.h>
#include <thrust/random.h>
#include <thrust/functional.h>
#include <iostream>
#include <vector>
#include <random>
#include <string>
#include <fstream>
#include <thread>
#include <atomic>
#include <mutex>
#include <cmath>
#include <algorithm>
#include <unordered_map>
#include <sstream>
#include <queue>
#include <memory>
#include <functional>
#include <filesystem>
#include <chrono>
#include <bit>
#include <array>
#include <tuple>
#include <utility>
#include <cstdint>
#include <curand_kernel.h>
#include <math_constants.h>

// See ref_harness.cu: the reference's global template swap is renamed.
#define swap ref_swap_
#include "cuda_libraries/types.h"

// Test image configuration (the reference fixes these at compile time in types.h).
#undef resolutionX
#undef resolutionY
#undef SAMPLES_PER_PIXEL
#undef MAX_RAY_RECURSION_DEPTH
#undef CHECK_SUBSURFACE_SCATTERING
#undef RENDER_MODE
#define resolutionX 48
#define resolutionY 48
#define SAMPLES_PER_PIXEL 32
#define MAX_RAY_RECURSION_DEPTH 8
#define CHECK_SUBSURFACE_SCATTERING false
#define RENDER_MODE PATH_TRACING

// include order of the reference's own mains (cornellBoxGuion.cu:1-22)
#include "shapes/Sphere.cu"
#include "shapes/Plane.cu"
#include "shapes/Triangle.cu"
#include "integration/Scene.cu"
#include "integration/PathTracerIntegrator.cu"
#include "integration/photonDispersion.cu"
#include "camera/ProjectiveCamera.cu"
#include "sampling/Sampler.cu"
#include "light/PointLight.cu"
#include "materials/LambertianMaterial.cu"
#include "materials/LightMaterial.cu"
#include "materials/GlassMaterial.cu"
#include "materials/MirrorMaterial.cu"
#include "materials/SSMaterial.cu"
#include "materials/PlasticUnrealMaterial.cu"
#include "textures/Texture.cu"
#include "textures/SphericalTexture.cu"
#include "cuda_libraries/FileImporting.cu"
#undef swap

#define REFR_API extern "C" __attribute__((visibility("default")))

namespace {
struct FilmPeek : public Film {
    using Film::pixelLight;
};
struct CameraPeek : public ProjectiveCamera {
    using ProjectiveCamera::rasterToCamera;
};
}  // namespace

REFR_API int refr_config(int *w, int *h, int *spp, int *depth)
{
    *w = resolutionX;
    *h = resolutionY;
    *spp = SAMPLES_PER_PIXEL;
    *depth = MAX_RAY_RECURSION_DEPTH;
    return 0;
}

// planes: per plane 12 floats (bottom-left corner, axisX, axisY, normal) as
// Plane(Point3f, Vector3f, Vector3f, Vector3f) (Plane.cu:26-50); kd: 3 floats per plane.
// out_mean: per-pixel mean radiance (Film sum / spp), row-major, 3 floats per pixel.
// out_c2w / out_r2c: the camera's cameraToWorld and rasterToCamera matrices (row-major).
// textured: nullable, per plane nonzero when its Lambertian material carries the Texture read
// from bmp_path (Texture::Texture, textures/Texture.cu); the plane's surface point is its
// object-space (x, y) (Plane.cu:82).
REFR_API int refr_render_tex(const char *obejota, int nplanes, const float *planes, const float *kd,
                             const char *bmp_path, const int *textured, float *out_mean, float *out_c2w,
                             float *out_r2c)
{
    std::unique_ptr<Texture> tex;
    if (bmp_path && textured) {
        try {
            tex.reset(new Texture(bmp_path));
        } catch (const std::exception &) {
            return 2;
        }
    }
    std::vector<Plane *> pl;
    std::vector<LambertianMaterial *> mats;
    std::vector<Shape *> shapes;
    for (int i = 0; i < nplanes; i++) {
        const float *p = planes + 12 * i;
        Plane *s = new Plane(Point3f(p[0], p[1], p[2]), Vector3f(p[3], p[4], p[5]), Vector3f(p[6], p[7], p[8]),
                             Vector3f(p[9], p[10], p[11]));
        LambertianMaterial *m = new LambertianMaterial(Spectrum(kd[3 * i], kd[3 * i + 1], kd[3 * i + 2]), Spectrum(0),
                                                       (tex && textured[i]) ? tex.get() : nullptr);
        s->setMaterial(m);
        pl.push_back(s);
        mats.push_back(m);
        shapes.push_back(s);
    }
    std::vector<Light *> lights;
    Camera *camera = nullptr;
    loadObejota(obejota, lights, shapes, camera);
    if (!camera) return 1;
    std::shared_ptr<std::vector<TriangleMesh>> meshes = std::make_shared<std::vector<TriangleMesh>>();
    std::vector<std::vector<Triangle>> triangles;
    Scene scene;
    scene.build(shapes, lights, triangles, meshes);
    PathTracerIntegrator integrator(camera);
    integrator.render(&scene);
    FilmPeek *film = static_cast<FilmPeek *>(camera->getFilm());
    for (int i = 0; i < resolutionX * resolutionY; i++) {
        out_mean[3 * i + 0] = (float)(film->pixelLight[i].getR() / SAMPLES_PER_PIXEL);
        out_mean[3 * i + 1] = (float)(film->pixelLight[i].getG() / SAMPLES_PER_PIXEL);
        out_mean[3 * i + 2] = (float)(film->pixelLight[i].getB() / SAMPLES_PER_PIXEL);
    }
    CameraPeek *pc = static_cast<CameraPeek *>(static_cast<ProjectiveCamera *>(camera));
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) {
            out_c2w[4 * r + c] = camera->cameraToWorld.getMatrix()[r][c];
            out_r2c[4 * r + c] = pc->rasterToCamera.getMatrix()[r][c];
        }
    for (auto *s : pl) delete s;
    for (auto *m : mats) delete m;
    return 0;
}

REFR_API int refr_render(const char *obejota, int nplanes, const float *planes, const float *kd, float *out_mean,
                         float *out_c2w, float *out_r2c)
{
    return refr_render_tex(obejota, nplanes, planes, kd, nullptr, nullptr, out_mean, out_c2w, out_r2c);
}

// SSMaterial::singleScattering (materials/SSMaterial.cu:108-181) of the reference's own class
// for n cases: wo, L 3 floats each; the sampler's generator is seeded with seeds[i] and its
// first sample (the one singleScattering draws) is returned in out_u. Out: value (3 floats),
// sampleDirection and outgoingPoint (3 floats each).
REFR_API int refr_single_scattering(float eta, float ns, float g, const float *sigma_s, const float *sigma_a,
                                    const float *wo, const float *L, const uint32_t *seeds, uint32_t n, float *out_rgb,
                                    float *out_wi, float *out_pt, float *out_u)
{
    SSMaterial m(Spectrum(0), Spectrum(0.5), Spectrum(0.1), eta, ns, nullptr, false,
                 Spectrum(sigma_s[0], sigma_s[1], sigma_s[2]), Spectrum(sigma_a[0], sigma_a[1], sigma_a[2]), g);
    for (uint32_t i = 0; i < n; i++) {
        Sampler s;
        s.rng = std::mt19937(seeds[i]);
        Sampler peek(s);
        out_u[i] = peek.get1Dsample();
        Vector3f wi;
        Point3f po;
        const Spectrum v = m.singleScattering(Vector3f(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), s, wi, Point2f(0, 0), po,
                                              Vector3f(L[3 * i], L[3 * i + 1], L[3 * i + 2]));
        out_rgb[3 * i] = (float)v.getR();
        out_rgb[3 * i + 1] = (float)v.getG();
        out_rgb[3 * i + 2] = (float)v.getB();
        out_wi[3 * i] = wi.x, out_wi[3 * i + 1] = wi.y, out_wi[3 * i + 2] = wi.z;
        out_pt[3 * i] = po.x, out_pt[3 * i + 1] = po.y, out_pt[3 * i + 2] = po.z;
    }
    return 0;
}

// Film accumulation files and computeRMSE (camera/Film.cu:366-449, 611-632) on films of the
// harness resolution. sum: 3 doubles per pixel (the per-pixel sums over `samples` samples).
namespace {
struct FilmFill : public Film {
    using Film::pixelLight;
    using Film::samplesComputedPixel0;
    using Film::samplesLoadedFromFile;
};
void fill(FilmFill &f, const double *sum, long long samples)
{
    for (int i = 0; i < resolutionX * resolutionY; i++) f.pixelLight[i] = Spectrum(sum[3 * i], sum[3 * i + 1], sum[3 * i + 2]);
    f.samplesComputedPixel0 = samples;
}
}  // namespace

REFR_API int refr_film_store(const char *path, const double *sum, long long samples)
{
    FilmFill f;
    fill(f, sum, samples);
    f.storeContributionsToFile(path);
    return 0;
}

REFR_API int refr_film_load(const char *path, double *sum, long long *samples)
{
    FilmFill f;
    if (!f.loadContributionsFromFile(path)) return 1;
    for (int i = 0; i < resolutionX * resolutionY; i++) {
        sum[3 * i] = f.pixelLight[i].getR();
        sum[3 * i + 1] = f.pixelLight[i].getG();
        sum[3 * i + 2] = f.pixelLight[i].getB();
    }
    *samples = f.samplesLoadedFromFile + f.samplesComputedPixel0;
    return 0;
}

// Film::writeToBMP / writeToPPM (camera/Film.cu:285-360): the reference's tone mapping of a
// film with these sums and its 8-bit image files (path without extension; the reference
// appends ".bmp" or ".ppm").
REFR_API int refr_film_write(const char *path, const double *sum, long long samples, int mode, int bmp)
{
    FilmFill f;
    fill(f, sum, samples);
    if (bmp)
        f.writeToBMP(path, (ToneMappingType)mode);
    else
        f.writeToPPM(path, (ToneMappingType)mode);
    return 0;
}

// BitmapImage::write_image (camera/BMP_Format.cu) of an image given in its own byte order:
// row i of image_bytes is row i of the file (bottom-up), BGR.
REFR_API int refr_bmp_write(const char *path, const unsigned char *bgr_rows, int width, int height)
{
    BitmapImage img(width, height);
    std::memcpy(img.image_bytes, bgr_rows, 3ull * width * height);
    std::ofstream file(path, std::ios::binary);
    img.write_image(file);
    return 0;
}

REFR_API double refr_film_rmse(const double *a, long long na, const double *b, long long nb)
{
    FilmFill fa, fb;
    fill(fa, a, na);
    fill(fb, b, nb);
    return computeRMSE(fa, fb);
}
