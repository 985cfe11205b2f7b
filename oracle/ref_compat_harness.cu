// Test infrastructure only: the reference's own scene objects — Plane shapes, Lambertian
// materials, and the camera, film and point lights read by its .obejota loader
// (cuda_libraries/FileImporting.cu:466) — rendered by this repository's GPU core through
// include/rt_b200_compat.hpp, the drop-in for Scene::build and PathTracerIntegrator::render
// (integration/Scene.cu:56-95, integration/PathTracerIntegrator.cu:140-210). The scene setup
// mirrors ref_render_harness.cu, which renders the same objects with the reference's own
// integrator; the image-parity test compares the two.
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
#include "materials/PlainMaterial.cu"
#include "materials/PhongMaterial.cu"
#include "materials/TrowbridgeMaterial.cu"
#include "materials/TrowbridgeBasicMaterial.cu"
#include "materials/BeckmannMaterial.cu"
#include "materials/FresnelBlendMaterial.cu"
#include "textures/Texture.cu"
#include "textures/SphericalTexture.cu"
#include "cuda_libraries/FileImporting.cu"
#undef swap

#include "../include/rt_b200_compat.hpp"

#define REFC_API extern "C" __attribute__((visibility("default")))

namespace {
struct FilmPeek : public Film {
    using Film::pixelLight;
};
thread_local std::string g_error;
}  // namespace

REFC_API int refc_config(int *w, int *h, int *spp, int *depth)
{
    *w = resolutionX;
    *h = resolutionY;
    *spp = SAMPLES_PER_PIXEL;
    *depth = MAX_RAY_RECURSION_DEPTH;
    return 0;
}

REFC_API const char *refc_error() { return g_error.c_str(); }

// The drop-in layer's mapping of a reference material (rt_material_type numbering of `kind`:
// 8 Beckmann, 9 TrowbridgeBasic, 10 FresnelBlend with emission ke = kd, 11 PlasticUnreal,
// 1 Trowbridge) into `out`. Returns 0, or 1 when the layer does not map it.
REFC_API int refc_map_material(int kind, const float *kd, const float *eta, const float *k, float rx, float ry,
                               rt_material *out)
{
    const Spectrum s_kd(kd[0], kd[1], kd[2]), s_eta(eta[0], eta[1], eta[2]), s_k(k[0], k[1], k[2]);
    std::unique_ptr<Material> m;
    switch (kind) {
    case 1: m.reset(new TrowbridgeMaterial(s_kd, s_eta, s_k, rx, ry)); break;
    case 8: m.reset(new BeckmannMaterial(s_kd, s_eta, s_k, rx, ry)); break;
    case 9: m.reset(new TrowbridgeBasicMaterial(s_kd, s_eta, s_k, rx, ry)); break;
    case 10: m.reset(new FresnelBlendMaterial(Spectrum(0), Spectrum(1), Spectrum(0), s_kd, 1.5f, 1.f)); break;
    case 11: m.reset(new PlasticUnrealMaterial(s_kd, 1.5f)); break;
    default: return 1;
    }
    const Texture *tex = nullptr;
    return rtb::compat_detail::to_rt_material(m.get(), *out, &tex) ? 0 : 1;
}

// The drop-in layer's reading of a material built with the reference's own Texture (read from
// bmp_path): kind 0 Lambertian, 1 Trowbridge, 3 Plain, 5 Phong, 6 SSMaterial, 8 Beckmann, 9
// TrowbridgeBasic, 10 FresnelBlend. *has_texture = 1 when the layer reports the material's
// Texture for registration. Returns 0, 1 when the layer does not map the class, 2 when the
// file cannot be read, 3 for an unknown kind.
REFC_API int refc_map_textured(int kind, const char *bmp_path, rt_material *out, int *has_texture)
{
    std::unique_ptr<Texture> t;
    try {
        t.reset(new Texture(bmp_path));
    } catch (const std::exception &) {
        return 2;
    }
    const Spectrum kd(0.6, 0.5, 0.4), eta(0.2, 0.9, 1.1), k(3.9, 2.4, 2.2);
    std::unique_ptr<Material> m;
    switch (kind) {
    case 0: m.reset(new LambertianMaterial(kd, Spectrum(0), t.get())); break;
    case 1: m.reset(new TrowbridgeMaterial(kd, eta, k, 0.3f, 0.1f, t.get())); break;
    case 3: m.reset(new PlainMaterial(kd, Spectrum(0), t.get())); break;
    case 5: m.reset(new PhongMaterial(Spectrum(0), kd, Spectrum(0.2), Spectrum(0), 1.5f, 20.f, t.get())); break;
    case 6: m.reset(new SSMaterial(Spectrum(0), kd, Spectrum(0.2), 1.3f, 20.f, t.get(), false, Spectrum(1), Spectrum(0.1), 0.f)); break;
    case 8: m.reset(new BeckmannMaterial(kd, eta, k, 0.3f, 0.1f, t.get())); break;
    case 9: m.reset(new TrowbridgeBasicMaterial(kd, eta, k, 0.3f, 0.1f, t.get())); break;
    case 10: m.reset(new FresnelBlendMaterial(Spectrum(0), kd, Spectrum(0), Spectrum(0), 1.5f, 1.f, t.get())); break;
    default: return 3;
    }
    const Texture *tex = nullptr;
    if (!rtb::compat_detail::to_rt_material(m.get(), *out, &tex)) return 1;
    *has_texture = (tex == t.get()) ? 1 : 0;
    return 0;
}

// planes: 12 floats each, Plane(corner, axisX, axisY, normal); kd: 3 floats each. out_mean:
// the film's per-pixel sum / spp after rtb::PathTracerIntegrator::render. Returns 0, or 1
// with refc_error() set.
// bmp_path / textured (nullable): per plane nonzero when its material carries the reference's
// own Texture read from bmp_path.
REFC_API int refc_render_tex(const char *obejota, int nplanes, const float *planes, const float *kd,
                             const char *bmp_path, const int *textured, uint32_t seed, float *out_mean)
{
    std::vector<Plane *> pl;
    std::vector<LambertianMaterial *> mats;
    std::vector<Shape *> shapes;
    std::unique_ptr<Texture> tex;
    int rc = 0;
    try {
        if (bmp_path && textured) tex.reset(new Texture(bmp_path));
        for (int i = 0; i < nplanes; i++) {
            const float *p = planes + 12 * i;
            Plane *s = new Plane(Point3f(p[0], p[1], p[2]), Vector3f(p[3], p[4], p[5]), Vector3f(p[6], p[7], p[8]),
                                 Vector3f(p[9], p[10], p[11]));
            LambertianMaterial *m = new LambertianMaterial(Spectrum(kd[3 * i], kd[3 * i + 1], kd[3 * i + 2]),
                                                           Spectrum(0), (tex && textured[i]) ? tex.get() : nullptr);
            s->setMaterial(m);
            pl.push_back(s);
            mats.push_back(m);
            shapes.push_back(s);
        }
        std::vector<Light *> lights;
        Camera *camera = nullptr;
        loadObejota(obejota, lights, shapes, camera);
        if (!camera) throw std::runtime_error("no camera in the scene file");
        std::shared_ptr<std::vector<TriangleMesh>> meshes = std::make_shared<std::vector<TriangleMesh>>();
        std::vector<std::vector<Triangle>> triangles;
        rtb::Scene scene(0);
        scene.build(shapes, lights, triangles, meshes);  // was: Scene::build
        rtb::PathTracerIntegrator integrator(camera, RT_RENDER_COMPAT, seed);
        integrator.render(&scene);                        // was: PathTracerIntegrator::render
        FilmPeek *film = static_cast<FilmPeek *>(camera->getFilm());
        for (int i = 0; i < resolutionX * resolutionY; i++) {
            out_mean[3 * i + 0] = (float)(film->pixelLight[i].getR() / SAMPLES_PER_PIXEL);
            out_mean[3 * i + 1] = (float)(film->pixelLight[i].getG() / SAMPLES_PER_PIXEL);
            out_mean[3 * i + 2] = (float)(film->pixelLight[i].getB() / SAMPLES_PER_PIXEL);
        }
    } catch (const std::exception &e) {
        g_error = e.what();
        rc = 1;
    }
    for (auto *s : pl) delete s;
    for (auto *m : mats) delete m;
    return rc;
}

REFC_API int refc_render(const char *obejota, int nplanes, const float *planes, const float *kd, uint32_t seed,
                         float *out_mean)
{
    return refc_render_tex(obejota, nplanes, planes, kd, nullptr, nullptr, seed, out_mean);
}
