// Test infrastructure only: a C-ABI shim that compiles the reference renderer's
// OWN headers (hsunekichi/2023_render_engine, included from the reference tree by
// the recipe in oracle/Makefile; nothing is copied) and exposes the pieces of
// its hot path that the parity tests and the CPU baseline need:
//
//   * the reference BVH exactly as BVH::BVH builds it (cuda_libraries/BVH.cu:314-341):
//     triangle bounds, scene bound reduced from Bound3f() (Triangle.cu:742-746),
//     Morton codes (Triangle.cu:718-734, geometricMath.cu:17-44), a sort of
//     (code, id) pairs (Triangle.cu:759-775), leaf init (BVH.cu:125-134),
//     BVH::generateHierarchy (BVH.cu:153-201) and computeBoundingBoxes (BVH.cu:203-212);
//   * BVH::intersectRay (BVH.cu:355-448) and BVH::intersectBruteForce (BVH.cu:452-476),
//     run on host threads;
//   * Triangle::intersects (Triangle.cu:434-643) for single-triangle checks;
//   * Sphere::intersects (Sphere.cu:357-398);
//   * the photon-map kd-tree nn::KDTree<Photon,3,PhotonPosition> (cuda_libraries/kdtree.h)
//     build and nearest_neighbors.
//
// Only tests, __graft_entry__.smoke() and bench.py's reference / cpu_baseline legs
// load the library built from this file. The product never links it.
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

// The reference declares a global `template swap(T&,T&)` (cuda_libraries/math.cu:56-63)
// that is ambiguous with thrust's and libstdc++'s when their headers are parsed after it.
// All system headers are included above, so renaming the token only affects the
// reference's own declaration and its own call sites.
#define swap ref_swap_
#include "cuda_libraries/BVH.cu"
#include "shapes/Sphere.cu"
#include "shapes/Plane.cu"
#include "cuda_libraries/kdtree.h"
#include "materials/LambertianMaterial.cu"
#include "materials/GlassMaterial.cu"
#include "materials/PhongMaterial.cu"
#include "materials/TrowbridgeMaterial.cu"
#include "materials/TrowbridgeBasicMaterial.cu"
#include "materials/BeckmannMaterial.cu"
#include "materials/FresnelBlendMaterial.cu"
#include "materials/PlasticUnrealMaterial.cu"
#undef swap

#define REFO_API extern "C" __attribute__((visibility("default")))

namespace {

struct RefBvh {
    std::vector<Point3f> vertices;
    TriangleMeshData mesh;
    std::vector<Triangle> triangles;
    thrust::host_vector<BVH::Node> nodes;
    thrust::host_vector<unsigned int> codes;
    thrust::host_vector<unsigned int> sortedIds;
    unsigned int root = 0;
};

template <typename F>
void parallel_for(uint64_t n, int nthreads, F &&f)
{
    if (nthreads <= 1 || n < 1024) {
        for (uint64_t i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> th;
    std::atomic<uint64_t> next(0);
    const uint64_t chunk = 4096;
    for (int t = 0; t < nthreads; t++) {
        th.emplace_back([&]() {
            for (;;) {
                uint64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                uint64_t e = std::min(n, b + chunk);
                for (uint64_t i = b; i < e; i++) f(i);
            }
        });
    }
    for (auto &t : th) t.join();
}

inline Ray make_ray(const float *o, const float *d, float tmax)
{
    return Ray(Point3f(o[0], o[1], o[2]), Vector3f(d[0], d[1], d[2]), tmax);
}

}  // namespace

// Builds the reference BVH over one triangle soup (vertex xyz array + 3 indices per
// triangle, in the order the reference concatenates meshes, BVH.cu:288-291).
// Requires ntri >= 2: generateHierarchy reads an empty FIFO when there is one triangle.
REFO_API void *refo_bvh_build(const float *xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri,
                              const uint8_t *transparent)
{
    if (ntri < 2) return nullptr;
    RefBvh *b = new RefBvh();
    b->vertices.resize(nv);
    for (uint32_t i = 0; i < nv; i++) b->vertices[i] = Point3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    b->mesh.vertices = b->vertices.data();
    b->triangles.resize(ntri);
    for (uint32_t t = 0; t < ntri; t++) {
        int vi[3] = {(int)idx[3 * t], (int)idx[3 * t + 1], (int)idx[3 * t + 2]};
        Triangle tri(vi);
        tri.mesh = &b->mesh;
        tri.meshId = 0;
        tri.isTransparent = transparent ? (transparent[t] != 0) : false;
        b->triangles[t] = tri;
    }
    // sort_by_morton (Triangle.cu:737-776), on the host.
    Bound3f world = Bound3f();
    for (uint32_t t = 0; t < ntri; t++) world = world + triangleWorldBoundFunctor()(b->triangles[t]);
    Morton3DFunctor morton(world);
    std::vector<std::pair<unsigned int, unsigned int>> keyed(ntri);
    for (uint32_t t = 0; t < ntri; t++) keyed[t] = {morton(b->triangles[t]), t};
    std::sort(keyed.begin(), keyed.end());
    b->codes.resize(ntri);
    b->sortedIds.resize(ntri);
    for (uint32_t t = 0; t < ntri; t++) {
        b->codes[t] = keyed[t].first;
        b->sortedIds[t] = keyed[t].second;
    }
    // generateTree (BVH.cu:216-234) with the reference's own member functions.
    b->nodes = thrust::host_vector<BVH::Node>(2 * ntri - 1);
    for (uint32_t i = 0; i < ntri; i++)
        BVH::initializeLeaf(i, b->nodes.data(), b->triangles.data(), b->sortedIds.data());
    // generateHierarchy/computeBoundingBoxes touch no BVH member; the BVH constructor
    // itself needs device memory, so they are invoked on raw storage.
    alignas(BVH) static unsigned char storage[sizeof(BVH)];
    BVH *shell = reinterpret_cast<BVH *>(storage);
    b->root = shell->generateHierarchy(b->codes, b->sortedIds, b->nodes, ntri);
    shell->computeBoundingBoxes(b->nodes, ntri);
    return b;
}

REFO_API void refo_bvh_free(void *h) { delete static_cast<RefBvh *>(h); }

REFO_API uint32_t refo_bvh_root(void *h) { return static_cast<RefBvh *>(h)->root; }

// Exports the reference tree: per node its box (pMin xyz, pMax xyz), objectId
// (-1 for interior nodes), children; plus the sorted Morton codes and ids.
REFO_API void refo_bvh_export(void *h, float *boxes, int32_t *objectIds, uint32_t *left, uint32_t *right,
                              uint32_t *codes, uint32_t *sortedIds)
{
    RefBvh *b = static_cast<RefBvh *>(h);
    size_t nn = b->nodes.size();
    size_t nt = b->triangles.size();
    for (size_t i = 0; i < nn; i++) {
        const BVH::Node &n = b->nodes[i];
        boxes[6 * i + 0] = n.boundingBox.pMin.x;
        boxes[6 * i + 1] = n.boundingBox.pMin.y;
        boxes[6 * i + 2] = n.boundingBox.pMin.z;
        boxes[6 * i + 3] = n.boundingBox.pMax.x;
        boxes[6 * i + 4] = n.boundingBox.pMax.y;
        boxes[6 * i + 5] = n.boundingBox.pMax.z;
        objectIds[i] = n.objectId;
        left[i] = n.isLeaf() ? 0xffffffffu : n.leftChild;
        right[i] = n.isLeaf() ? 0xffffffffu : n.rightChild;
    }
    for (size_t i = 0; i < nt; i++) {
        codes[i] = b->codes[i];
        sortedIds[i] = b->sortedIds[i];
    }
}

// BVH::intersectRay over a batch of rays (SoA origin/direction, tMax per ray).
REFO_API void refo_bvh_intersect(void *h, const float *o, const float *d, const float *tmax, uint64_t n,
                                 int checkShadow, int32_t *out, int nthreads)
{
    RefBvh *b = static_cast<RefBvh *>(h);
    const BVH::Node *nodes = b->nodes.data();
    const Triangle *tris = b->triangles.data();
    unsigned int root = b->root;
    parallel_for(n, nthreads, [&](uint64_t i) {
        Ray r = make_ray(o + 3 * i, d + 3 * i, tmax ? tmax[i] : INFINITY);
        out[i] = BVH::intersectRay(r, root, nodes, tris, checkShadow != 0);
    });
}

// BVH::intersectBruteForce (leaf-box prefilter, then every triangle in sorted order).
REFO_API void refo_bvh_brute(void *h, const float *o, const float *d, const float *tmax, uint64_t n,
                             int checkShadow, int32_t *out, int nthreads)
{
    RefBvh *b = static_cast<RefBvh *>(h);
    const BVH::Node *nodes = b->nodes.data();
    const Triangle *tris = b->triangles.data();
    int nt = (int)b->triangles.size();
    parallel_for(n, nthreads, [&](uint64_t i) {
        Ray r = make_ray(o + 3 * i, d + 3 * i, tmax ? tmax[i] : INFINITY);
        out[i] = BVH::intersectBruteForce(r, tris, nodes, nt, checkShadow != 0);
    });
}

// Triangle::intersects for triangle `tri` of the soup: returns 1/0 and updates
// *hitOffset exactly as the reference does (including its update before the
// error-bound rejection, Triangle.cu:569-593).
REFO_API int refo_triangle_intersects(void *h, uint32_t tri, const float *o, const float *d, float tmax,
                                      float *hitOffset, int checkShadow)
{
    RefBvh *b = static_cast<RefBvh *>(h);
    Ray r = make_ray(o, d, tmax);
    Float off = *hitOffset;
    bool hit = b->triangles[tri].intersects(r, off, checkShadow != 0);
    *hitOffset = off;
    return hit ? 1 : 0;
}

// Distance to the hit of the reference's tie-free closest triangle, via Triangle::intersect
// (the full-interaction version, Triangle.cu:162-431); returns -1 when it reports no hit.
REFO_API void refo_triangle_hit_t(void *h, const int32_t *ids, const float *o, const float *d, uint64_t n,
                                  float *tOut, int nthreads)
{
    RefBvh *b = static_cast<RefBvh *>(h);
    parallel_for(n, nthreads, [&](uint64_t i) {
        tOut[i] = -1.0f;
        if (ids[i] < 0) return;
        Ray r = make_ray(o + 3 * i, d + 3 * i, INFINITY);
        Float off = INFINITY;
        if (b->triangles[ids[i]].intersects(r, off, false)) tOut[i] = off;
    });
}

namespace {
struct RefSpheres {
    std::vector<Sphere *> spheres;
    std::vector<Material *> materials;
    ~RefSpheres()
    {
        for (auto *s : spheres) delete s;
        for (auto *m : materials) delete m;
    }
};
}  // namespace

// Spheres built with the reference's Sphere(Point3f center, Float radius) constructor
// (Sphere.cu:233-245: translate(center) * rotateZ(90)); glass=1 makes it transparent
// for shadow rays like GlassMaterial (DielectricMaterial.cu isTransparent()).
REFO_API void *refo_spheres_build(const float *centers, const float *radii, const uint8_t *glass, uint32_t n)
{
    RefSpheres *s = new RefSpheres();
    for (uint32_t i = 0; i < n; i++) {
        Sphere *sp = new Sphere(Point3f(centers[3 * i], centers[3 * i + 1], centers[3 * i + 2]), radii[i]);
        Material *m = (glass && glass[i]) ? (Material *)new GlassMaterial(Spectrum(1.0))
                                          : (Material *)new LambertianMaterial(Spectrum(0.8));
        sp->setMaterial(m);
        s->spheres.push_back(sp);
        s->materials.push_back(m);
    }
    return s;
}

REFO_API void refo_spheres_free(void *h) { delete static_cast<RefSpheres *>(h); }

// Both matrices the reference stores for sphere i (row-major 4x4, objectToWorld then worldToObject).
REFO_API void refo_sphere_matrices(void *h, uint32_t i, float *o2w, float *w2o)
{
    RefSpheres *s = static_cast<RefSpheres *>(h);
    struct Peek : public Sphere {
        using Sphere::objectToWorld;
        using Sphere::worldToObject;
    };
    Peek *p = static_cast<Peek *>(s->spheres[i]);
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) {
            o2w[4 * r + c] = p->objectToWorld.m[r][c];
            w2o[4 * r + c] = p->worldToObject.m[r][c];
        }
}

// Closest sphere hit in the order Scene::intersects loops shapes (Scene.cu:134-139):
// each Sphere::intersects lowers the running offset; returns the last sphere that did.
REFO_API void refo_spheres_intersect(void *h, const float *o, const float *d, uint64_t n, int checkShadow,
                                     int32_t *outId, float *outT, int nthreads)
{
    RefSpheres *s = static_cast<RefSpheres *>(h);
    parallel_for(n, nthreads, [&](uint64_t i) {
        Ray r = make_ray(o + 3 * i, d + 3 * i, INFINITY);
        Float off = INFINITY;
        int id = -1;
        for (size_t j = 0; j < s->spheres.size(); j++)
            if (s->spheres[j]->intersects(r, off, checkShadow != 0)) id = (int)j;
        outId[i] = id;
        outT[i] = off;
    });
}

namespace {
struct RefPlanes {
    std::vector<Plane *> planes;
    std::vector<Material *> materials;
    ~RefPlanes()
    {
        for (auto *p : planes) delete p;
        for (auto *m : materials) delete m;
    }
};
}  // namespace

// Planes built with the reference's Plane(bottomLeftCorner, axisX, axisY, normal) constructor
// (Plane.cu:26-50), 12 floats each; glass=1 makes one transparent for shadow rays.
REFO_API void *refo_planes_build(const float *p12, const uint8_t *glass, uint32_t n)
{
    RefPlanes *s = new RefPlanes();
    for (uint32_t i = 0; i < n; i++) {
        const float *p = p12 + 12 * i;
        Plane *pl = new Plane(Point3f(p[0], p[1], p[2]), Vector3f(p[3], p[4], p[5]), Vector3f(p[6], p[7], p[8]),
                              Vector3f(p[9], p[10], p[11]));
        Material *m = (glass && glass[i]) ? (Material *)new GlassMaterial(Spectrum(1.0))
                                          : (Material *)new LambertianMaterial(Spectrum(0.8));
        pl->setMaterial(m);
        s->planes.push_back(pl);
        s->materials.push_back(m);
    }
    return s;
}

REFO_API void refo_planes_free(void *h) { delete static_cast<RefPlanes *>(h); }

// Both matrices the reference stores for plane i (row-major 4x4, objectToWorld then worldToObject).
REFO_API void refo_plane_matrices(void *h, uint32_t i, float *o2w, float *w2o)
{
    struct Peek : public Plane {
        using Plane::objectToWorld;
        using Plane::worldToObject;
    };
    Peek *p = static_cast<Peek *>(static_cast<RefPlanes *>(h)->planes[i]);
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) {
            o2w[4 * r + c] = p->objectToWorld.m[r][c];
            w2o[4 * r + c] = p->worldToObject.m[r][c];
        }
}

// Scene::intersects' shape loop (Scene.cu:141-146) over these planes, starting from the offset
// in t_inout (INFINITY, or a triangle hit's offset): each Plane::intersects that lowers the
// running offset replaces the hit. outId: the last plane that did (-1: none).
REFO_API void refo_planes_intersect(void *h, const float *o, const float *d, uint64_t n, int checkShadow,
                                    int32_t *outId, float *t_inout, int nthreads)
{
    RefPlanes *s = static_cast<RefPlanes *>(h);
    parallel_for(n, nthreads, [&](uint64_t i) {
        Ray r = make_ray(o + 3 * i, d + 3 * i, INFINITY);
        Float off = t_inout[i];
        int id = -1;
        for (size_t j = 0; j < s->planes.size(); j++)
            if (s->planes[j]->intersects(r, off, checkShadow != 0)) id = (int)j;
        outId[i] = id;
        t_inout[i] = off;
    });
}

namespace {
struct RefPhotonMap {
    PhotonMap *map = nullptr;
    ~RefPhotonMap() { delete map; }
};
}  // namespace

// Builds the reference photon kd-tree (kdtree.h:78-108) over photon locations; the
// photon's own index is carried in its radiance (R channel) so queries can report it.
REFO_API void *refo_kdtree_build(const float *pos, const int32_t *shapeIds, uint64_t n)
{
    std::vector<Photon> ph(n);
    for (uint64_t i = 0; i < n; i++) {
        ph[i].location = Point3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        ph[i].shapeId = shapeIds ? shapeIds[i] : -1;
        ph[i].radiance = Spectrum((double)i, 0.0, 0.0);
    }
    RefPhotonMap *m = new RefPhotonMap();
    m->map = new PhotonMap(ph);
    return m;
}

REFO_API void refo_kdtree_free(void *h) { delete static_cast<RefPhotonMap *>(h); }

// nearest_neighbors (kdtree.h:161-197) per query: up to k photon indices (heap order
// as the reference returns them) with their count.
REFO_API void refo_kdtree_knn(void *h, const float *q, const int32_t *qShape, uint64_t nq, uint32_t k,
                              float radius, int32_t *outIdx, uint32_t *outCount, int nthreads)
{
    RefPhotonMap *m = static_cast<RefPhotonMap *>(h);
    parallel_for(nq, nthreads, [&](uint64_t i) {
        Point3f p(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
        int sid = qShape ? qShape[i] : -1;
        std::vector<Photon> r = m->map->nearest_neighbors(p, (unsigned long)k, radius, sid);
        uint32_t c = (uint32_t)std::min<size_t>(r.size(), k);
        outCount[i] = c;
        for (uint32_t j = 0; j < k; j++) outIdx[(uint64_t)i * k + j] = j < c ? (int32_t)r[j].radiance.getR() : -1;
    });
}

REFO_API int refo_version() { return 1; }


// diffusionTermBSSRDF (cuda_libraries/geometricMath.cu:500-522) for one photon: out = Sd (rgb).
// camera: point, direction to the camera, shading normal; photon: location, incoming ray
// direction, surface normal.
REFO_API void refo_diffusion_term(const float *cam_p, const float *cam_dir, const float *cam_n, const float *ph_loc,
                                  const float *ph_dir, const float *ph_n, const float *sigma_s, const float *sigma_a,
                                  float g, float eta, double *out)
{
    Photon ph(Ray(Point3f(ph_loc[0], ph_loc[1], ph_loc[2]), Vector3f(ph_dir[0], ph_dir[1], ph_dir[2])),
              Point3f(ph_loc[0], ph_loc[1], ph_loc[2]), Vector3f(ph_n[0], ph_n[1], ph_n[2]), Spectrum(1), 0,
              Point2f(0, 0));
    Spectrum s = diffusionTermBSSRDF(Point3f(cam_p[0], cam_p[1], cam_p[2]), Vector3f(cam_dir[0], cam_dir[1], cam_dir[2]),
                                     Vector3f(cam_n[0], cam_n[1], cam_n[2]), ph,
                                     Spectrum(sigma_s[0], sigma_s[1], sigma_s[2]),
                                     Spectrum(sigma_a[0], sigma_a[1], sigma_a[2]), g, eta);
    out[0] = s.getR();
    out[1] = s.getG();
    out[2] = s.getB();
}

// Material::lightReflected and ::pdf of the reference's own classes in shading space for n
// direction pairs: kind 0 Lambertian, 1 Trowbridge, 8 Beckmann, 9 TrowbridgeBasic,
// 10 FresnelBlend, 11 PlasticUnreal (the rt_material_type numbers); out_f 3 floats per pair.
REFO_API int refo_material_eval(int kind, const float *kd, const float *eta, const float *k, float rx, float ry,
                                const float *wo, const float *wi, uint32_t n, float *out_f, float *out_pdf)
{
    const Spectrum s_kd(kd[0], kd[1], kd[2]), s_eta(eta[0], eta[1], eta[2]), s_k(k[0], k[1], k[2]);
    std::unique_ptr<Material> m;
    switch (kind) {
    case 0: m.reset(new LambertianMaterial(s_kd)); break;
    case 1: m.reset(new TrowbridgeMaterial(s_kd, s_eta, s_k, rx, ry)); break;
    case 8: m.reset(new BeckmannMaterial(s_kd, s_eta, s_k, rx, ry)); break;
    case 9: m.reset(new TrowbridgeBasicMaterial(s_kd, s_eta, s_k, rx, ry)); break;
    case 10: m.reset(new FresnelBlendMaterial(Spectrum(0), s_kd, s_k, Spectrum(0), 1.5f, 1.f)); break;
    case 11: m.reset(new PlasticUnrealMaterial(s_kd, 1.5f)); break;
    default: return 1;
    }
    for (uint32_t i = 0; i < n; i++) {
        Vector3f o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        Spectrum f = m->lightReflected(o, w, Point2f(0, 0));
        out_f[3 * i] = (float)f.getR();
        out_f[3 * i + 1] = (float)f.getG();
        out_f[3 * i + 2] = (float)f.getB();
        out_pdf[i] = m->pdf(o, w);
    }
    return 0;
}

// Texture::getColor (textures/Texture.cu:179-192) of the reference's own Texture, loaded by
// its own BMP reader (Texture::loadBmpImage) from `bmp_path`, at n surface points (2 floats
// each); out_rgb 3 floats per point. Returns 1 when the file cannot be read.
REFO_API int refo_texture_lookup(const char *bmp_path, const float *uv, uint32_t n, float *out_rgb)
{
    std::unique_ptr<Texture> t;
    try {
        t.reset(new Texture(bmp_path));
    } catch (const std::exception &) {
        return 1;
    }
    for (uint32_t i = 0; i < n; i++) {
        const Spectrum c = t->getColor(Point2f(uv[2 * i], uv[2 * i + 1]));
        out_rgb[3 * i] = (float)c.getR();
        out_rgb[3 * i + 1] = (float)c.getG();
        out_rgb[3 * i + 2] = (float)c.getB();
    }
    return 0;
}

// Material::lightReflected and ::pdf of the reference's classes built with a Texture (read
// from `bmp_path` as above), each direction pair i evaluated at surface point uv[i]: kind 0
// Lambertian, 1 Trowbridge, 5 Phong (kd, ks = eta, ns = rx), 8 Beckmann, 9 TrowbridgeBasic.
REFO_API int refo_material_eval_tex(int kind, const float *kd, const float *eta, const float *k, float rx, float ry,
                                    const char *bmp_path, const float *uv, const float *wo, const float *wi,
                                    uint32_t n, float *out_f, float *out_pdf)
{
    std::unique_ptr<Texture> t;
    try {
        t.reset(new Texture(bmp_path));
    } catch (const std::exception &) {
        return 1;
    }
    const Spectrum s_kd(kd[0], kd[1], kd[2]), s_eta(eta[0], eta[1], eta[2]), s_k(k[0], k[1], k[2]);
    std::unique_ptr<Material> m;
    switch (kind) {
    case 0: m.reset(new LambertianMaterial(s_kd, Spectrum(0), t.get())); break;
    case 1: m.reset(new TrowbridgeMaterial(s_kd, s_eta, s_k, rx, ry, t.get())); break;
    case 5: m.reset(new PhongMaterial(Spectrum(0), s_kd, s_eta, Spectrum(0), 1.5f, rx, t.get())); break;
    case 8: m.reset(new BeckmannMaterial(s_kd, s_eta, s_k, rx, ry, t.get())); break;
    case 9: m.reset(new TrowbridgeBasicMaterial(s_kd, s_eta, s_k, rx, ry, t.get())); break;
    default: return 2;
    }
    for (uint32_t i = 0; i < n; i++) {
        Vector3f o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        Spectrum f = m->lightReflected(o, w, Point2f(uv[2 * i], uv[2 * i + 1]));
        out_f[3 * i] = (float)f.getR();
        out_f[3 * i + 1] = (float)f.getG();
        out_f[3 * i + 2] = (float)f.getB();
        out_pdf[i] = m->pdf(o, w);
    }
    return 0;
}

// PhongMaterial::lightReflected and ::pdf (materials/PhongMaterial.cu:70-100) in shading space
// for n direction pairs: out_f 3 floats per pair, out_pdf 1.
REFO_API void refo_phong_eval(const float *kd, const float *ks, float ns, const float *wo, const float *wi, uint32_t n,
                              float *out_f, float *out_pdf)
{
    PhongMaterial m(Spectrum(0), Spectrum(kd[0], kd[1], kd[2]), Spectrum(ks[0], ks[1], ks[2]), Spectrum(0), 1.5f, ns);
    for (uint32_t i = 0; i < n; i++) {
        Vector3f o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        Spectrum f = m.lightReflected(o, w, Point2f(0, 0));
        out_f[3 * i] = (float)f.getR();
        out_f[3 * i + 1] = (float)f.getG();
        out_f[3 * i + 2] = (float)f.getB();
        out_pdf[i] = m.pdf(o, w);
    }
}
