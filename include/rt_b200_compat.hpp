/* rt_b200_compat.hpp — the reference renderer's own scene API on top of the C ABI (rt_b200.h).
 *
 * The reference (hsunekichi/2023_render_engine) is header-only C++: its programs include
 * shapes/, materials/, light/, camera/ and integration/ directly. Include this header after
 * those, in the same translation unit, and replace the hot-path calls:
 *
 *   rtb::Scene::build              for Scene::build               (integration/Scene.cu:56-95)
 *   rtb::Scene::intersects         for Scene::intersects          (integration/Scene.cu:108-150)
 *   rtb::PathTracerIntegrator      for PathTracerIntegrator       (integration/PathTracerIntegrator.cu:140-210)
 *   rtb::Scene::generatePhotons    for generatePhotons            (integration/photonDispersion.cu:175-192)
 *   rtb::Scene::search_nearest     for Scene::search_nearest      (integration/Scene.cu:704-722)
 *
 * The objects are the reference's own: Shape* (Sphere, Plane), the triangle lists and meshes
 * of its loaders, Light* (PointLight), Material* (Lambertian, Trowbridge, Dielectric/Glass,
 * Light, Mirror, Plain), Camera* (ProjectiveCamera) and its Film. Their protected members are
 * read through accessor subclasses declared below. Errors become std::runtime_error, the way
 * the reference reports them; a material or shape class the core does not implement is an
 * error (RT_ERR_UNSUPPORTED) rather than a silent substitute.
 */
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

#include "rt_b200.h"

namespace rtb {

inline void check(int status)
{
    if (status != RT_OK) {
        char msg[512];
        rt_last_error(msg, sizeof msg);
        throw std::runtime_error(std::string("rt_b200: ") + msg);
    }
}

namespace compat_detail {

// Accessors for protected members of the reference's classes (layout-identical subclasses).
struct SphereAccess : public Sphere {
    using Sphere::objectToWorld;
    using Sphere::sph_radius;
    using Sphere::worldToObject;
};
struct PlaneAccess : public Plane {
    using Plane::objectToWorld;
    using Plane::worldToObject;
};
struct LightMaterialAccess : public LightMaterial {
    using LightMaterial::color;
    using LightMaterial::intensity;
};
struct LightAccess : public Light {
    using Light::color;
    using Light::intensity;
};
struct CameraAccess : public ProjectiveCamera {
    using ProjectiveCamera::focalDistance;
    using ProjectiveCamera::lensRadius;
    using ProjectiveCamera::rasterToCamera;
};
struct FilmAccess : public Film {
    using Film::current_resolution;
};

inline void matrix16(const Transform &t, float out[16])
{
    const auto m = t.getMatrix();
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) out[4 * r + c] = (float)m[r][c];
}

inline void rgb(const Spectrum &s, float out[3])
{
    out[0] = (float)s.getR();
    out[1] = (float)s.getG();
    out[2] = (float)s.getB();
}

// Material* -> rt_material (materials/*.cu); false for a class the core does not implement.
// *tex receives the Texture the material reads (null: none); the caller registers it and sets
// o.texture.
inline bool to_rt_material(const Material *m, rt_material &o, const Texture **tex)
{
    o = rt_material{};
    *tex = nullptr;
    if (const auto *l = dynamic_cast<const LambertianMaterial *>(m)) {
        o.type = RT_MAT_LAMBERTIAN;
        rgb(l->bsdf.color, o.color);
        *tex = l->bsdf.texture;
    } else if (const auto *t = dynamic_cast<const TrowbridgeMaterial *>(m)) {
        o.type = RT_MAT_TROWBRIDGE;
        *tex = t->bsdf.text;
        rgb(t->bsdf.kd, o.color);
        rgb(t->bsdf.eta, o.eta);
        rgb(t->bsdf.k, o.k);
        // TrowbridgeBSDF keeps alpha = sqrt(roughness) (TrowbridgeBSDF.cu:56-59)
        o.roughness[0] = (float)(t->bsdf.alphaX * t->bsdf.alphaX);
        o.roughness[1] = (float)(t->bsdf.alphaY * t->bsdf.alphaY);
    } else if (const auto *tb = dynamic_cast<const TrowbridgeBasicMaterial *>(m)) {
        o.type = RT_MAT_TROWBRIDGE_BASIC;  // TrowbridgeBasicBSDF keeps alpha = sqrt(roughness) too
        *tex = tb->bsdf.text;
        rgb(tb->bsdf.kd, o.color);
        rgb(tb->bsdf.eta, o.eta);
        rgb(tb->bsdf.k, o.k);
        o.roughness[0] = (float)(tb->bsdf.alphaX * tb->bsdf.alphaX);
        o.roughness[1] = (float)(tb->bsdf.alphaY * tb->bsdf.alphaY);
    } else if (const auto *bk = dynamic_cast<const BeckmannMaterial *>(m)) {
        o.type = RT_MAT_BECKMANN;  // BeckmannBSDF: alpha = sqrt(roughness) (BeckmannBSDF.cu:30-37)
        *tex = bk->bsdf.text;
        rgb(bk->bsdf.kd, o.color);
        rgb(bk->bsdf.eta, o.eta);
        rgb(bk->bsdf.k, o.k);
        o.roughness[0] = (float)(bk->bsdf.alphaX * bk->bsdf.alphaX);
        o.roughness[1] = (float)(bk->bsdf.alphaY * bk->bsdf.alphaY);
    } else if (const auto *fb = dynamic_cast<const FresnelBlendMaterial *>(m)) {
        o.type = RT_MAT_FRESNEL_BLEND;  // kd = 1, ks = 0, alpha = 0.5 fixed by its constructor
        rgb(fb->ke, o.extra);
    } else if (const auto *pu = dynamic_cast<const PlasticUnrealMaterial *>(m)) {
        o.type = RT_MAT_PLASTIC;
        rgb(pu->kd, o.color);
    } else if (const auto *d = dynamic_cast<const DielectricMaterial *>(m)) {
        o.type = RT_MAT_DIELECTRIC;
        rgb(d->ks, o.color);
        o.ior = (float)d->ior;
    } else if (const auto *e = dynamic_cast<const LightMaterial *>(m)) {
        const auto *a = static_cast<const LightMaterialAccess *>(e);
        o.type = RT_MAT_LIGHT;
        rgb(a->color, o.color);
        o.intensity = (float)a->intensity;
    } else if (const auto *r = dynamic_cast<const MirrorMaterial *>(m)) {
        o.type = RT_MAT_MIRROR;
        rgb(r->color, o.color);
    } else if (const auto *p = dynamic_cast<const PlainMaterial *>(m)) {
        o.type = RT_MAT_PLAIN;
        *tex = p->texture;
        rgb(p->kd, o.color);
    } else if (const auto *ss = dynamic_cast<const SSMaterial *>(m)) {
        // Phong surface (SSMaterial.cu:29) over the dipole medium
        o.type = RT_MAT_SUBSURFACE;
        *tex = ss->text;
        rgb(ss->kd, o.color);
        rgb(ss->surfaceMaterial.ks, o.k);
        o.roughness[0] = (float)ss->surfaceMaterial.ns;
        o.roughness[1] = (float)ss->g;
        o.ior = (float)ss->eta;
        rgb(ss->sigmaS, o.eta);
        rgb(ss->sigmaA, o.extra);
    } else if (const auto *ph = dynamic_cast<const PhongMaterial *>(m)) {
        if (ph->ke.maxComponent() > 0) return false;  // emissive Phong: not implemented by the core
        o.type = RT_MAT_PHONG;
        *tex = ph->text;
        rgb(ph->kd, o.color);
        rgb(ph->ks, o.k);
        o.roughness[0] = (float)ph->ns;
    } else {
        return false;
    }
    if (m->isTransparent()) o.flags |= RT_MATF_TRANSPARENT;
    return true;
}

}  // namespace compat_detail

// The GPU scene: Scene::build's inputs uploaded to the core, plus the queries on them.
class Scene {
public:
    explicit Scene(int device = 0)
    {
        check(rt_context_create(device, &ctx_));
        int s = rt_scene_create(ctx_, &scene_);
        if (s != RT_OK) {
            rt_context_destroy(ctx_);
            check(s);
        }
    }
    ~Scene()
    {
        if (pmap_) rt_photon_map_destroy(pmap_);
        rt_scene_destroy(scene_);
        rt_context_destroy(ctx_);
    }
    Scene(const Scene &) = delete;
    Scene &operator=(const Scene &) = delete;

    // Scene::build (Scene.cu:56-95): shapes, lights and the loaders' triangle lists with host
    // copies of their meshes (the reference's Scene::copyMesh makes the same copies).
    // Triangle ids follow the same concatenation order as the reference's BVH.
    void build(const std::vector<Shape *> &shapes, const std::vector<Light *> &lights,
               std::vector<std::vector<Triangle>> &initTriangles, const std::vector<CpuTriangleMesh> &meshes)
    {
        if (initTriangles.size() > meshes.size()) throw std::runtime_error("rt_b200: a triangle list has no mesh");
        int32_t shape_id = 0;
        for (size_t i = 0; i < initTriangles.size(); i++, shape_id++) add_triangles(initTriangles[i], meshes[i], shape_id);
        for (size_t j = 0; j < shapes.size(); j++) add_shape(shapes[j], (int32_t)j);
        for (const Light *l : lights) add_light(l);
        check(rt_scene_set_materials(scene_, materials_.data(), (uint32_t)materials_.size()));
        if (!tri_material_.empty())
            check(rt_scene_set_triangle_materials(scene_, 0, (uint32_t)tri_material_.size(), tri_material_.data()));
        check(rt_scene_commit(scene_));
        shapes_ = shapes;
    }

    // The same with the loaders' device meshes (copied to the host first).
    void build(const std::vector<Shape *> &shapes, const std::vector<Light *> &lights,
               std::vector<std::vector<Triangle>> &initTriangles,
               std::shared_ptr<std::vector<TriangleMesh>> &triangleMesh)
    {
        std::vector<CpuTriangleMesh> host;
        if (!initTriangles.empty())
            for (const TriangleMesh &m : *triangleMesh) host.emplace_back(m);
        build(shapes, lights, initTriangles, host);
    }

    // Scene::intersects (Scene.cu:108-150): closest hit over triangles and shapes; true on a
    // hit, with hitOffset its distance. `prim` gets the triangle id, or RT_PRIM_SHAPE | index.
    bool intersects(const Ray &ray, Float &hitOffset, int32_t *prim = nullptr) const
    {
        rt_ray r{(float)ray.origin.x, (float)ray.origin.y, (float)ray.origin.z, (float)ray.maximumOffset,
                 (float)ray.direction.x, (float)ray.direction.y, (float)ray.direction.z, 0u};
        rt_hit h;
        check(rt_trace_closest_host(scene_, &r, 1, &h, 0));
        if (prim) *prim = h.prim;
        if (h.prim < 0) return false;
        hitOffset = h.t;
        return true;
    }

    // generatePhotons (photonDispersion.cu:175-192) + Scene::buildPhotonStructures: traces
    // nPhotons from the point lights and builds the kd-tree gather structure.
    void generatePhotons(uint64_t nPhotons, uint32_t maxDepth, uint32_t seed = 0, bool compat = true,
                         uint32_t k = 100, float radius = 100.f)
    {
        if (pmap_) {
            rt_photon_map_destroy(pmap_);
            pmap_ = nullptr;
        }
        rt_photon_trace_stats st;
        check(rt_photons_trace(scene_, nPhotons, maxDepth, 3, seed, compat ? RT_RENDER_COMPAT : 0u, &pmap_, &st));
        check(rt_photon_map_build(pmap_));
        check(rt_render_set_photon_map(scene_, pmap_, k, radius));  // MAX_NEIGHBOURS, PHOTON_SEARCH_RADIUS
        photons_.resize(0);
    }

    // Scene::search_nearest (Scene.cu:704-722): the photons among the k nearest within
    // `radius` that lie on shape `shapeId` (-1: any), as the reference's Photon objects.
    std::vector<Photon> search_nearest(Point3f position, Float radius, unsigned long k, int shapeId = -1) const
    {
        if (!pmap_) throw std::runtime_error("Photon map not built");
        if (k == 0 || k > 128) throw std::runtime_error("rt_b200: search_nearest takes 1 <= k <= 128");
        load_photons();
        // the k-NN call works on device buffers
        float q[3] = {(float)position.x, (float)position.y, (float)position.z};
        int32_t sid = shapeId;
        float *dq = nullptr;
        int32_t *ds = nullptr, *didx = nullptr;
        uint32_t *dcnt = nullptr;
        check_cuda(cudaMalloc(&dq, sizeof q));
        check_cuda(cudaMalloc(&ds, sizeof sid));
        check_cuda(cudaMalloc(&didx, sizeof(int32_t) * k));
        check_cuda(cudaMalloc(&dcnt, sizeof(uint32_t)));
        std::vector<int32_t> idx(k);
        uint32_t cnt = 0;
        int s = RT_OK;
        if (cudaMemcpy(dq, q, sizeof q, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(ds, &sid, sizeof sid, cudaMemcpyHostToDevice) != cudaSuccess)
            s = RT_ERR_CUDA;
        if (s == RT_OK)
            s = rt_photon_knn(pmap_, dq, shapeId >= 0 ? ds : nullptr, 1, (uint32_t)k, (float)radius,
                              didx, nullptr, dcnt);
        if (s == RT_OK && (cudaMemcpy(&cnt, dcnt, sizeof cnt, cudaMemcpyDeviceToHost) != cudaSuccess ||
                           cudaMemcpy(idx.data(), didx, sizeof(int32_t) * k, cudaMemcpyDeviceToHost) != cudaSuccess))
            s = RT_ERR_CUDA;
        cudaFree(dq);
        cudaFree(ds);
        cudaFree(didx);
        cudaFree(dcnt);
        if (s == RT_ERR_CUDA) throw std::runtime_error("rt_b200: search_nearest: CUDA copy failed");
        check(s);
        std::vector<Photon> out;
        for (uint32_t i = 0; i < cnt; i++) {
            const rt_photon &p = photons_[(size_t)idx[i]];
            const Point3f at(p.pos[0], p.pos[1], p.pos[2]);
            out.emplace_back(Ray(at, Vector3f(p.dir[0], p.dir[1], p.dir[2])), at,
                             Vector3f(p.normal[0], p.normal[1], p.normal[2]),
                             Spectrum(p.power[0], p.power[1], p.power[2]), p.shape_id, Point2f(0, 0));
        }
        return out;
    }

    rt_scene *handle() const { return scene_; }
    rt_context *context() const { return ctx_; }
    rt_photon_map *photon_map() const { return pmap_; }

private:
    static void check_cuda(cudaError_t e)
    {
        if (e != cudaSuccess) throw std::runtime_error(std::string("rt_b200: ") + cudaGetErrorString(e));
    }

    uint32_t material_index(const Material *m)
    {
        for (size_t i = 0; i < material_ptrs_.size(); i++)
            if (material_ptrs_[i] == m) return (uint32_t)i;
        rt_material rm;
        const Texture *tex = nullptr;
        if (!m || !compat_detail::to_rt_material(m, rm, &tex))
            check_unsupported(std::string("material class ") + (m ? typeid(*m).name() : "(null)"));
        if (tex) rm.texture = 1u + texture_index(tex);
        material_ptrs_.push_back(m);
        materials_.push_back(rm);
        return (uint32_t)(materials_.size() - 1);
    }

    // a Texture's texels, read through Texture::getColor at the texel centres (its pixelMatrix
    // is not public), registered once per Texture object
    uint32_t texture_index(const Texture *t)
    {
        for (size_t i = 0; i < texture_ptrs_.size(); i++)
            if (texture_ptrs_[i] == t) return texture_ids_[i];
        const uint32_t w = t->getWidth(), h = t->getHeight();
        std::vector<float> rgb(3ull * w * h);
        for (uint32_t y = 0; y < h; y++)
            for (uint32_t x = 0; x < w; x++) {
                const Spectrum c = t->getColor(Point2f(((float)x + 0.5f) / (float)w, ((float)y + 0.5f) / (float)h));
                float *o = rgb.data() + 3ull * ((size_t)y * w + x);
                compat_detail::rgb(c, o);
            }
        uint32_t id = 0;
        check(rt_scene_add_texture(scene_, rgb.data(), w, h, &id));
        texture_ptrs_.push_back(t);
        texture_ids_.push_back(id);
        return id;
    }

    [[noreturn]] static void check_unsupported(const std::string &what)
    {
        throw std::runtime_error("rt_b200: unsupported " + what + " (RT_ERR_UNSUPPORTED)");
    }

    void add_triangles(const std::vector<Triangle> &tris, const CpuTriangleMesh &mesh, int32_t shape_id)
    {
        if (tris.empty()) return;
        std::vector<float> xyz(3 * mesh.vertices.size());
        for (size_t v = 0; v < mesh.vertices.size(); v++) {
            xyz[3 * v] = (float)mesh.vertices[v].x;
            xyz[3 * v + 1] = (float)mesh.vertices[v].y;
            xyz[3 * v + 2] = (float)mesh.vertices[v].z;
        }
        std::vector<float> nrm(3 * mesh.normals.size());
        for (size_t v = 0; v < mesh.normals.size(); v++) {
            nrm[3 * v] = (float)mesh.normals[v].x;
            nrm[3 * v + 1] = (float)mesh.normals[v].y;
            nrm[3 * v + 2] = (float)mesh.normals[v].z;
        }
        std::vector<uint32_t> idx(3 * tris.size()), nidx;
        if (!mesh.normals.empty()) nidx.resize(3 * tris.size());
        // texture coordinates per triangle through its textureIndices (Triangle.cu:134-151)
        std::vector<float> uv;
        if (!mesh.textureCoords.empty()) uv.resize(6 * tris.size());
        const uint32_t first = (uint32_t)tri_material_.size();
        bool transparent = false;
        for (size_t t = 0; t < tris.size(); t++) {
            for (int k = 0; k < 3; k++) {
                idx[3 * t + k] = tris[t].vertexIndices[k];
                if (!nidx.empty()) nidx[3 * t + k] = tris[t].normalIndices[k];
                if (!uv.empty()) {
                    const Point2f &c = mesh.textureCoords[tris[t].textureIndices[k]];
                    uv[6 * t + 2 * k] = (float)c.x;
                    uv[6 * t + 2 * k + 1] = (float)c.y;
                }
            }
            transparent = transparent || tris[t].isTransparent;
            tri_material_.push_back(material_index(tris[t].material));
        }
        check(rt_scene_add_mesh(scene_, xyz.data(), (uint32_t)mesh.vertices.size(), idx.data(), (uint32_t)tris.size(),
                                nrm.empty() ? nullptr : nrm.data(), (uint32_t)mesh.normals.size(),
                                nidx.empty() ? nullptr : nidx.data(), tri_material_.back(), shape_id, transparent,
                                nullptr));
        if (!uv.empty()) check(rt_scene_set_triangle_uvs(scene_, first, (uint32_t)tris.size(), uv.data()));
    }

    void add_shape(const Shape *s, int32_t index)
    {
        const uint32_t mat = material_index(s->getMaterial());
        const bool transparent = s->getMaterial()->isTransparent();
        if (const auto *sp = dynamic_cast<const Sphere *>(s)) {
            const auto *a = static_cast<const compat_detail::SphereAccess *>(sp);
            float o2w[16], w2o[16];
            compat_detail::matrix16(a->objectToWorld, o2w);
            compat_detail::matrix16(a->worldToObject, w2o);
            check(rt_scene_add_sphere(scene_, o2w, w2o, (float)a->sph_radius, mat, index, transparent, nullptr));
        } else if (const auto *pl = dynamic_cast<const Plane *>(s)) {
            // the reference's own plane: its matrices and Plane::intersects' arithmetic
            const auto *a = static_cast<const compat_detail::PlaneAccess *>(pl);
            float o2w[16], w2o[16];
            compat_detail::matrix16(a->objectToWorld, o2w);
            compat_detail::matrix16(a->worldToObject, w2o);
            check(rt_scene_add_plane(scene_, o2w, w2o, mat, index, transparent, nullptr));
        } else {
            check_unsupported(std::string("shape class ") + typeid(*s).name());
        }
    }

    void add_light(const Light *l)
    {
        if (!dynamic_cast<const PointLight *>(l)) check_unsupported(std::string("light class ") + typeid(*l).name());
        const auto *a = static_cast<const compat_detail::LightAccess *>(l);
        const Point3f p = l->getPosition();
        const float pos[3] = {(float)p.x, (float)p.y, (float)p.z};
        float c[3];
        compat_detail::rgb(a->color, c);
        check(rt_scene_add_point_light(scene_, pos, c, (float)a->intensity));
    }

    void load_photons() const
    {
        if (!photons_.empty()) return;
        uint64_t n = 0;
        check(rt_photon_map_count(pmap_, &n));
        photons_.resize(n);
        if (n) check(rt_photon_map_get(pmap_, 0, n, photons_.data()));
    }

    rt_context *ctx_ = nullptr;
    rt_scene *scene_ = nullptr;
    rt_photon_map *pmap_ = nullptr;
    std::vector<const Material *> material_ptrs_;
    std::vector<rt_material> materials_;
    std::vector<const Texture *> texture_ptrs_;
    std::vector<uint32_t> texture_ids_;
    std::vector<uint32_t> tri_material_;
    std::vector<Shape *> shapes_;
    mutable std::vector<rt_photon> photons_;
};

// The estimator flags of the reference's compile-time configuration (types.h): its quirks,
// CHECK_SUBSURFACE_SCATTERING and RENDER_MODE (PHOTON_MAPPING and HYBRID need the photon map of
// Scene::generatePhotons).
inline uint32_t reference_flags()
{
    uint32_t f = RT_RENDER_COMPAT;
    if (CHECK_SUBSURFACE_SCATTERING) f |= RT_RENDER_SUBSURFACE;
    if (RENDER_MODE == PHOTON_MAPPING) f |= RT_RENDER_PHOTON_MAP;
    if (RENDER_MODE == HYBRID) f |= RT_RENDER_HYBRID;
    return f;
}

// PathTracerIntegrator (PathTracerIntegrator.cu:140-210): renders the camera's film with
// SAMPLES_PER_PIXEL samples and MAX_RAY_RECURSION_DEPTH bounces (the reference's compile-time
// configuration), adding each pixel's sum over its samples to the Film as the reference does
// (Film::addSample, NaN/Inf samples replaced by the mean of the valid ones,
// pathTracing.cu:457-490). `flags` selects the estimator (RT_RENDER_COMPAT: the reference's).
class PathTracerIntegrator {
public:
    explicit PathTracerIntegrator(Camera *camera, uint32_t flags = RT_RENDER_COMPAT, uint32_t seed = 0)
        : camera_(camera), flags_(flags), seed_(seed)
    {
    }

    void render(Scene *scene, uint32_t spp = SAMPLES_PER_PIXEL, uint32_t maxDepth = MAX_RAY_RECURSION_DEPTH)
    {
        const auto *cam = dynamic_cast<const ProjectiveCamera *>(camera_);
        if (!cam) throw std::runtime_error("rt_b200: unsupported camera class (RT_ERR_UNSUPPORTED)");
        const auto *ca = static_cast<const compat_detail::CameraAccess *>(cam);
        Film *film = camera_->getFilm();
        const auto *fa = static_cast<const compat_detail::FilmAccess *>(film);
        rt_camera rc{};
        compat_detail::matrix16(camera_->cameraToWorld, rc.camera_to_world);
        compat_detail::matrix16(ca->rasterToCamera, rc.raster_to_camera);
        rc.lens_radius = (float)ca->lensRadius;
        rc.focal_distance = (float)ca->focalDistance;
        rc.width = fa->current_resolution.x;
        rc.height = fa->current_resolution.y;
        const size_t npix = (size_t)rc.width * rc.height;
        float *sum = nullptr;
        uint32_t *count = nullptr;
        if (cudaMalloc(&sum, 12 * npix) != cudaSuccess) throw std::runtime_error("rt_b200: out of device memory");
        if (cudaMalloc(&count, 4 * npix) != cudaSuccess) {
            cudaFree(sum);
            throw std::runtime_error("rt_b200: out of device memory");
        }
        std::vector<float> hsum(3 * npix);
        std::vector<uint32_t> hcount(npix);
        int s = (cudaMemset(sum, 0, 12 * npix) == cudaSuccess && cudaMemset(count, 0, 4 * npix) == cudaSuccess)
                    ? RT_OK
                    : RT_ERR_CUDA;
        rt_render_opts o{spp, sample_offset_, maxDepth, 3, seed_, flags_, 0, 0};
        rt_render_stats st{};
        if (s == RT_OK) s = rt_render(scene->handle(), &rc, &o, sum, count, nullptr, &st);
        if (s == RT_OK && (cudaMemcpy(hsum.data(), sum, 12 * npix, cudaMemcpyDeviceToHost) != cudaSuccess ||
                           cudaMemcpy(hcount.data(), count, 4 * npix, cudaMemcpyDeviceToHost) != cudaSuccess))
            s = RT_ERR_CUDA;
        cudaFree(sum);
        cudaFree(count);
        if (s == RT_ERR_CUDA) throw std::runtime_error("rt_b200: render: CUDA copy failed");
        check(s);
        for (uint32_t y = 0; y < rc.height; y++)
            for (uint32_t x = 0; x < rc.width; x++) {
                const size_t i = (size_t)y * rc.width + x;
                const double scale = hcount[i] ? (double)spp / hcount[i] : 0.0;
                film->addSample(Point2i(x, y), Spectrum(hsum[3 * i] * scale, hsum[3 * i + 1] * scale, hsum[3 * i + 2] * scale),
                                (int)spp);
            }
        sample_offset_ += spp;
        stats_ = st;
    }

    const rt_render_stats &stats() const { return stats_; }

private:
    Camera *camera_;
    uint32_t flags_, seed_;
    uint32_t sample_offset_ = 0;  // successive calls continue the sample sequence
    rt_render_stats stats_{};
};

}  // namespace rtb
