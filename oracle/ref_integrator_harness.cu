// Test and baseline infrastructure only: the reference renderer's OWN integrator
// (PathTracerIntegrator::render, integration/PathTracerIntegrator.cu:140-210, with its bounce
// loop computeSamples, pathTracing.cu:284-414, and Scene::build, Scene.cu:56-95) on scenes
// given as triangle meshes, spheres and planes, compiled from its sources where they lie.
//
// The same file is compiled twice (oracle/Makefile):
//
//  * libref_integrator_host.so: thrust's device system set to OpenMP
//    (THRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_OMP, a configuration thrust documents). Every
//    thrust::device_vector of the reference then lives in host memory and every thrust
//    algorithm it runs (the Morton sort of its BVH build, the BVH traversal of
//    BVH::intersectRaysGpu) runs on the host cores, so the reference's whole render runs on
//    the CPU, triangle meshes included. This is the reference's host-compiled integrator:
//    IEEE host arithmetic, its own 128 worker threads for shading, OpenMP threads for its
//    traversal. No device code runs.
//  * libref_integrator_cuda.so: the stock CUDA build with the flags of the reference's
//    compile.sh (-O3 --use_fast_math -maxrregcount=64): its BVH is built and traversed on the
//    GPU through thrust, shading runs on its host threads. This is the reference's CUDA build.
//
// The reference fixes resolution, samples per pixel and depth at compile time (types.h:41-74);
// here those macros name variables set by refi_config before a render. Rays are counted at
// the reference's two BVH call sites in Scene.cu (extension rays at :184, shadow rays at :119)
// by a macro that adds a counter call in front of each call and leaves the call itself as it
// is. Used by tests and bench.py only; the product never links it.
//
// REFI_HOST_BACKEND selects the OpenMP device system for the host compilation pass only:
// thrust's OpenMP backend is host code, and the device pass (which compiles the reference's
// __device__ functions and kernels, none of which the render launches) keeps the CUDA system.
#if defined(REFI_HOST_BACKEND) && !defined(__CUDA_ARCH__)
#define THRUST_DEVICE_SYSTEM THRUST_DEVICE_SYSTEM_OMP
// the device pass instantiates thrust's CUDA kernels from the same host code; their host-side
// stubs (never launched) need the CUDA backend's declarations in this pass too
#include <thrust/system/cuda/vector.h>
#include <thrust/system/cuda/execution_policy.h>
#include <thrust/system/cuda/detail/copy.h>
#include <thrust/system/cuda/detail/fill.h>
#include <thrust/system/cuda/detail/for_each.h>
#include <thrust/system/cuda/detail/parallel_for.h>
#include <thrust/system/cuda/detail/reduce.h>
#include <thrust/system/cuda/detail/sequence.h>
#include <thrust/system/cuda/detail/sort.h>
#include <thrust/system/cuda/detail/tabulate.h>
#include <thrust/system/cuda/detail/transform.h>
#include <thrust/system/cuda/detail/uninitialized_copy.h>
#include <thrust/system/cuda/detail/uninitialized_fill.h>
#include <cub/cub.cuh>
#endif
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

namespace refi {
// Render configuration read by the reference's compile-time macros below.
struct Config {
    int w = 64, h = 64, spp = 4, depth = 8;
    unsigned photons = 100000;  // N_PHOTON_SAMPLES of a photon pass
    int mode = 0;               // RENDER_MODE: 0 PATH_TRACING, 1 PHOTON_MAPPING, 2 HYBRID
    bool subsurface = false;    // CHECK_SUBSURFACE_SCATTERING
    unsigned neighbours = 100;  // MAX_NEIGHBOURS
    float radius = 100.f;       // PHOTON_SEARCH_RADIUS
};
Config g_cfg;
std::atomic<unsigned long long> g_ext_rays{0}, g_shadow_rays{0};
// Counts the rays of one BVH call; the first argument is the host vector of rays.
template <class V, class... Rest>
int count_extension(const V &rays, const Rest &...)
{
    g_ext_rays += rays.size();
    return 0;
}
template <class V, class... Rest>
int count_shadow(const V &rays, const Rest &...)
{
    g_shadow_rays += rays.size();
    return 0;
}
}  // namespace refi

// See ref_harness.cu: the reference's global template swap is renamed.
#define swap ref_swap_
#include "cuda_libraries/types.h"

#undef resolutionX
#undef resolutionY
#undef SAMPLES_PER_PIXEL
#undef MAX_RAY_RECURSION_DEPTH
#undef CHECK_SUBSURFACE_SCATTERING
#undef RENDER_MODE
#undef N_PHOTON_SAMPLES
#undef MAX_NEIGHBOURS
#undef PHOTON_SEARCH_RADIUS
#ifdef __CUDA_ARCH__
#define N_PHOTON_SAMPLES 1
#define MAX_NEIGHBOURS 100
#define PHOTON_SEARCH_RADIUS 100
#define CHECK_SUBSURFACE_SCATTERING false
#define RENDER_MODE PATH_TRACING
// device pass: the reference's __device__ code that names these is never launched here
#define resolutionX 640
#define resolutionY 360
#define SAMPLES_PER_PIXEL 1
#define MAX_RAY_RECURSION_DEPTH 1
#else
#define resolutionX (refi::g_cfg.w)
#define resolutionY (refi::g_cfg.h)
#define SAMPLES_PER_PIXEL (refi::g_cfg.spp)
#define MAX_RAY_RECURSION_DEPTH (refi::g_cfg.depth)
#define N_PHOTON_SAMPLES (refi::g_cfg.photons)
#define MAX_NEIGHBOURS (refi::g_cfg.neighbours)
#define PHOTON_SEARCH_RADIUS (refi::g_cfg.radius)
#define CHECK_SUBSURFACE_SCATTERING (refi::g_cfg.subsurface)
#define RENDER_MODE ((RenderMode)refi::g_cfg.mode)
#endif

// include order of the reference's own mains (cornellBoxGuion.cu:1-22); its BVH first, so
// that the counting macro below applies to Scene.cu's call sites only
#include "shapes/Sphere.cu"
#include "shapes/Plane.cu"
#include "shapes/Triangle.cu"
#include "cuda_libraries/BVH.cu"
// Scene.cu calls `bvh->intersectRays(rays, ...)` with 4 arguments for shadow rays (:119) and
// with 2 for extension rays (:184). The expansion keeps that call (a macro does not expand
// itself again) and puts a counter call before it in the same expression statement.
#define REFI_PICK(_1, _2, _3, _4, NAME, ...) NAME
#define REFI_EXT(...) getRoot(), refi::count_extension(__VA_ARGS__), bvh->intersectRays(__VA_ARGS__)
#define REFI_SHADOW(...) getRoot(), refi::count_shadow(__VA_ARGS__), bvh->intersectRays(__VA_ARGS__)
#define intersectRays(...) REFI_PICK(__VA_ARGS__, REFI_SHADOW, REFI_SHADOW, REFI_EXT, REFI_EXT)(__VA_ARGS__)
#include "integration/Scene.cu"
#undef intersectRays
#include "integration/PathTracerIntegrator.cu"
#include "integration/photonDispersion.cu"
#include "camera/ProjectiveCamera.cu"
#include "sampling/Sampler.cu"
#include "light/PointLight.cu"
#include "materials/LambertianMaterial.cu"
#include "materials/LightMaterial.cu"
#include "materials/GlassMaterial.cu"
#include "materials/MirrorMaterial.cu"
#include "materials/TrowbridgeMaterial.cu"
#include "materials/SSMaterial.cu"
#include "materials/PlasticUnrealMaterial.cu"
#include "textures/Texture.cu"
#include "textures/SphericalTexture.cu"
#include "cuda_libraries/FileImporting.cu"
#undef swap

#define REFI_API extern "C" __attribute__((visibility("default")))

namespace {
struct FilmPeek : public Film {
    using Film::pixelLight;
};
struct CameraPeek : public ProjectiveCamera {
    using ProjectiveCamera::rasterToCamera;
};
struct ScenePeek : public Scene {
    using Scene::photons;
};
thread_local std::string g_error;

// Material table entry: 16 floats.
//   [0] kind: 0 Lambertian (kd = [1..3]), 1 Trowbridge (kd [1..3], eta [4..6], k [7..9],
//       roughness x [10], y [11]), 2 Light (color [1..3], intensity [4]), 3 Dielectric
//       (color [1..3], ior [4]), 4 Mirror (color [1..3]), 5 SSMaterial (kd [1..3], ks [4..6],
//       eta [7], ns [8], sigma_s [9..11], sigma_a [12..14], g [15])
constexpr int kEntry = 16;
Material *make_material(const float *m)
{
    const Spectrum c(m[1], m[2], m[3]);
    switch ((int)m[0]) {
    case 5:
        return new SSMaterial(Spectrum(0), c, Spectrum(m[4], m[5], m[6]), m[7], m[8], nullptr, false,
                              Spectrum(m[9], m[10], m[11]), Spectrum(m[12], m[13], m[14]), m[15]);
    case 0:
        return new LambertianMaterial(c);
    case 1:
        return new TrowbridgeMaterial(c, Spectrum(m[4], m[5], m[6]), Spectrum(m[7], m[8], m[9]), m[10], m[11]);
    case 2:
        return new LightMaterial(c, m[4]);
    case 3:
        return new DielectricMaterial(c, m[4]);
    case 4:
        return new MirrorMaterial(c);
    default:
        return nullptr;
    }
}
}  // namespace

REFI_API const char *refi_error() { return g_error.c_str(); }

// 1 when this library runs the reference's thrust work on the host (OpenMP device system).
REFI_API int refi_host_backend()
{
#if THRUST_DEVICE_SYSTEM == THRUST_DEVICE_SYSTEM_OMP
    return 1;
#else
    return 0;
#endif
}

REFI_API int refi_config(int w, int h, int spp, int depth)
{
    if (w <= 0 || h <= 0 || spp <= 0 || depth <= 0) return 1;
    refi::g_cfg.w = w, refi::g_cfg.h = h, refi::g_cfg.spp = spp, refi::g_cfg.depth = depth;
    return 0;
}

// The photon-mapping settings of types.h:51-60: RENDER_MODE (0 path tracing, 1 photon mapping,
// 2 hybrid), CHECK_SUBSURFACE_SCATTERING, N_PHOTON_SAMPLES, MAX_NEIGHBOURS, PHOTON_SEARCH_RADIUS.
REFI_API int refi_config_photons(int mode, int subsurface, unsigned photons, unsigned neighbours, float radius)
{
    if (mode < 0 || mode > 2 || photons == 0 || neighbours == 0) return 1;
    refi::g_cfg.mode = mode, refi::g_cfg.subsurface = subsurface != 0, refi::g_cfg.photons = photons;
    refi::g_cfg.neighbours = neighbours, refi::g_cfg.radius = radius;
    return 0;
}

// Renders with the reference's integrator.
//   obejota: path of a scene file holding the camera and point lights (read by the reference's
//            own loadObejota, FileImporting.cu:466);
//   triangles: nv vertices (xyz), ntri triangles (3 indices, its material and its shape id,
//            the reference's meshId), one TriangleMesh;
//   spheres: center xyz + radius per sphere (Sphere(Point3f, Float), Sphere.cu:233) and its
//            material; planes: 12 floats per plane as Plane(corner, axisX, axisY, normal),
//            Plane.cu:26-50, and its material;
//   materials: nmat entries of 16 floats (make_material).
// out_mean: per-pixel mean radiance (the Film's sum / spp), row-major, 3 floats per pixel.
// out_c2w / out_r2c (nullable): the camera's cameraToWorld and rasterToCamera (row-major).
// out_stats (nullable): [0] seconds in PathTracerIntegrator::render, [1] extension rays,
//   [2] shadow rays, [3] seconds in Scene::build (the reference's BVH build).
namespace {
// The reference's scene objects for one call; owns what the reference leaves to its caller.
struct SceneInput {
    std::vector<std::unique_ptr<Material>> mats;
    std::vector<std::unique_ptr<Shape>> owned;
    std::vector<Shape *> shapes;
    std::vector<Light *> lights;
    Camera *camera = nullptr;
    std::shared_ptr<std::vector<TriangleMesh>> meshes = std::make_shared<std::vector<TriangleMesh>>();
    std::vector<std::vector<Triangle>> triangles;
    ~SceneInput()
    {
        for (Light *l : lights) delete l;
    }
};

// Fills `in` from the arrays refi_render documents; 0 or 1 with g_error set.
int make_scene_input(SceneInput &in, const char *obejota, uint32_t nv, const float *xyz, uint32_t ntri,
                     const uint32_t *idx, const uint32_t *tri_mat, const int32_t *tri_shape, uint32_t nspheres,
                     const float *spheres, const uint32_t *sphere_mat, uint32_t nplanes, const float *planes,
                     const uint32_t *plane_mat, uint32_t nmat, const float *materials)
{
    for (uint32_t i = 0; i < nmat; i++) {
        in.mats.emplace_back(make_material(materials + kEntry * i));
        if (!in.mats.back()) return g_error = "unknown material kind", 1;
    }
    for (uint32_t i = 0; i < nspheres; i++) {
        const float *sp = spheres + 4 * i;
        if (sphere_mat[i] >= nmat) return g_error = "sphere material", 1;
        Sphere *sh = new Sphere(Point3f(sp[0], sp[1], sp[2]), sp[3]);
        sh->setMaterial(in.mats[sphere_mat[i]].get());
        in.owned.emplace_back(sh);
        in.shapes.push_back(sh);
    }
    for (uint32_t i = 0; i < nplanes; i++) {
        const float *p = planes + 12 * i;
        if (plane_mat[i] >= nmat) return g_error = "plane material", 1;
        Plane *pl = new Plane(Point3f(p[0], p[1], p[2]), Vector3f(p[3], p[4], p[5]), Vector3f(p[6], p[7], p[8]),
                              Vector3f(p[9], p[10], p[11]));
        pl->setMaterial(in.mats[plane_mat[i]].get());
        in.owned.emplace_back(pl);
        in.shapes.push_back(pl);
    }
    loadObejota(obejota, in.lights, in.shapes, in.camera);
    if (ntri > 0) {
        TriangleMesh mesh;
        thrust::host_vector<Point3f> hv(nv);
        for (uint32_t i = 0; i < nv; i++) hv[i] = Point3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        mesh.vertices = hv;
        std::vector<Triangle> tris(ntri);
        for (uint32_t t = 0; t < ntri; t++) {
            if (tri_mat[t] >= nmat) return g_error = "triangle material", 1;
            Triangle face;
            face.meshId = tri_shape ? tri_shape[t] : 0;
            for (int k = 0; k < 3; k++) face.vertexIndices[k] = idx[3 * t + k];
            face.setMaterial(in.mats[tri_mat[t]].get());
            tris[t] = face;
        }
        in.meshes->push_back(mesh);
        in.triangles.push_back(tris);
    }
    return 0;
}
}  // namespace

REFI_API int refi_render(const char *obejota, uint32_t nv, const float *xyz, uint32_t ntri, const uint32_t *idx,
                         const uint32_t *tri_mat, const int32_t *tri_shape, uint32_t nspheres, const float *spheres,
                         const uint32_t *sphere_mat, uint32_t nplanes, const float *planes, const uint32_t *plane_mat,
                         uint32_t nmat, const float *materials, float *out_mean, float *out_c2w, float *out_r2c,
                         double *out_stats)
{
    try {
        SceneInput in;
        if (make_scene_input(in, obejota, nv, xyz, ntri, idx, tri_mat, tri_shape, nspheres, spheres, sphere_mat,
                             nplanes, planes, plane_mat, nmat, materials))
            return 1;
        Camera *camera = in.camera;
        if (!camera) return g_error = "no camera in the scene file", 1;
        refi::g_ext_rays = 0;
        refi::g_shadow_rays = 0;
        auto t0 = std::chrono::steady_clock::now();
        Scene scene;
        scene.build(in.shapes, in.lights, in.triangles, in.meshes);
        auto t1 = std::chrono::steady_clock::now();
        PathTracerIntegrator integrator(camera);
        std::streambuf *old = std::cout.rdbuf(nullptr);  // the integrator prints progress lines
        integrator.render(&scene);
        std::cout.rdbuf(old);
        auto t2 = std::chrono::steady_clock::now();
        FilmPeek *film = static_cast<FilmPeek *>(camera->getFilm());
        const int npix = resolutionX * resolutionY;
        for (int i = 0; i < npix; i++) {
            out_mean[3 * i + 0] = (float)(film->pixelLight[i].getR() / SAMPLES_PER_PIXEL);
            out_mean[3 * i + 1] = (float)(film->pixelLight[i].getG() / SAMPLES_PER_PIXEL);
            out_mean[3 * i + 2] = (float)(film->pixelLight[i].getB() / SAMPLES_PER_PIXEL);
        }
        if (out_c2w && out_r2c) {
            CameraPeek *pc = static_cast<CameraPeek *>(static_cast<ProjectiveCamera *>(camera));
            for (int r = 0; r < 4; r++)
                for (int c = 0; c < 4; c++) {
                    out_c2w[4 * r + c] = camera->cameraToWorld.getMatrix()[r][c];
                    out_r2c[4 * r + c] = pc->rasterToCamera.getMatrix()[r][c];
                }
        }
        if (out_stats) {
            out_stats[0] = std::chrono::duration<double>(t2 - t1).count();
            out_stats[1] = (double)refi::g_ext_rays.load();
            out_stats[2] = (double)refi::g_shadow_rays.load();
            out_stats[3] = std::chrono::duration<double>(t1 - t0).count();
        }
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

// The reference's photon pass, generatePhotons (photonDispersion.cu:175-192: Scene::generatePhotons,
// Scene.cu:989-1018, then computePhotons), with `nphotons` emitted photons on the scene
// refi_render takes (the scene file supplies the point lights; a camera in it is optional).
// Out: the stored photons, up to cap: location (3 floats), radiance (3 floats, the reference's
// double spectrum rounded to float) and shape id per photon, and their number (*count, which may
// exceed cap).
REFI_API int refi_photons(const char *obejota, uint32_t nv, const float *xyz, uint32_t ntri, const uint32_t *idx,
                          const uint32_t *tri_mat, const int32_t *tri_shape, uint32_t nspheres, const float *spheres,
                          const uint32_t *sphere_mat, uint32_t nplanes, const float *planes, const uint32_t *plane_mat,
                          uint32_t nmat, const float *materials, uint32_t nphotons, float *out_pos, float *out_power,
                          int32_t *out_shape, uint64_t cap, uint64_t *count)
{
    try {
        SceneInput in;
        if (make_scene_input(in, obejota, nv, xyz, ntri, idx, tri_mat, tri_shape, nspheres, spheres, sphere_mat,
                             nplanes, planes, plane_mat, nmat, materials))
            return 1;
        refi::g_cfg.photons = nphotons;
        ScenePeek scene;
        scene.build(in.shapes, in.lights, in.triangles, in.meshes);
        Sampler sampler;
        generatePhotons(&scene, &sampler);
        const auto &ph = scene.photons;
        *count = ph.size();
        for (uint64_t i = 0; i < ph.size() && i < cap; i++) {
            const Photon &p = ph[i];
            out_pos[3 * i] = p.location.x, out_pos[3 * i + 1] = p.location.y, out_pos[3 * i + 2] = p.location.z;
            out_power[3 * i] = (float)p.radiance.getR();
            out_power[3 * i + 1] = (float)p.radiance.getG();
            out_power[3 * i + 2] = (float)p.radiance.getB();
            out_shape[i] = p.shapeId;
        }
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

// Material::sampleDirection of the reference's own class (make_material's table entry) for n
// shading-frame directions wo (3 floats each). Case i seeds the reference's sampler with
// seeds[i]; out_u receives its first 1D sample (the dielectric's lobe choice). Out: the sampled
// direction (3 floats; left at 0 where the reference leaves it unset) and the returned value
// (3 floats).
REFI_API int refi_material_sample(const float *entry, const float *wo, const uint32_t *seeds, uint32_t n,
                                  float *out_wi, float *out_value, float *out_u)
{
    std::unique_ptr<Material> m(make_material(entry));
    if (!m) return g_error = "unknown material kind", 1;
    for (uint32_t i = 0; i < n; i++) {
        Sampler s;
        s.rng = std::mt19937(seeds[i]);
        Sampler peek(s);
        out_u[i] = peek.get1Dsample();
        Vector3f wi(0, 0, 0);
        Point3f po;
        const Spectrum v = m->sampleDirection(Vector3f(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), s, wi, Point2f(0, 0), po,
                                              Vector3f(0, 0, 0));
        out_wi[3 * i] = wi.x, out_wi[3 * i + 1] = wi.y, out_wi[3 * i + 2] = wi.z;
        out_value[3 * i] = (float)v.getR();
        out_value[3 * i + 1] = (float)v.getG();
        out_value[3 * i + 2] = (float)v.getB();
    }
    return 0;
}
