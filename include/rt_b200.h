/*
 * rt_b200.h — C ABI of the B200 rendering core.
 *
 * One GPU (sm_100a). Plain pointers and sizes only; every function returns an
 * rt_status (0 = RT_OK). rt_last_error() returns the message of the last failure
 * on the calling host thread. Calls on one rt_context are serialised by the
 * caller (the reference API is not re-entrant either, cuda_libraries/types.h:20);
 * work is queued on the context's stream and functions return once it is done
 * unless stated otherwise.
 *
 * Each entry point names the reference interface it replaces
 * (hsunekichi/2023_render_engine, path:line).
 */
#ifndef RT_B200_H
#define RT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: rt_material gained `texture` (76 bytes); a caller built against 1 passes 72-byte entries */
#define RT_B200_ABI_VERSION 2

#if defined(__GNUC__)
#define RT_API __attribute__((visibility("default")))
#else
#define RT_API
#endif

typedef enum rt_status {
    RT_OK = 0,
    RT_ERR_INVALID = 1,     /* bad argument (null pointer, size, index) */
    RT_ERR_CUDA = 2,        /* CUDA runtime error */
    RT_ERR_OOM = 3,         /* device allocation failed */
    RT_ERR_TIMEOUT = 4,     /* a device loop hit its iteration cap */
    RT_ERR_UNSUPPORTED = 5, /* feature or material not supported */
    RT_ERR_STATE = 6,       /* wrong call order (e.g. trace before commit) */
    RT_ERR_CAPACITY = 7     /* a fixed-capacity queue or buffer would overflow */
} rt_status;

typedef struct rt_context rt_context;
typedef struct rt_scene rt_scene;

/* ---------------------------------------------------------------- basics */

RT_API int rt_abi_version(void);
/* Copies the calling thread's last error message (NUL-terminated, truncated). */
RT_API int rt_last_error(char *buf, size_t len);

/* Selects the device (replaces the bare cudaSetDevice(argv[2]) of the reference
 * mains, cornellBoxGuion.cu:35-49) and creates the context's stream. */
RT_API int rt_context_create(int device, rt_context **out);
RT_API int rt_context_destroy(rt_context *ctx);
/* Use a caller-owned cudaStream_t (passed as void*) instead of the internal one. */
RT_API int rt_context_set_stream(rt_context *ctx, void *cuda_stream);
RT_API int rt_context_synchronize(rt_context *ctx);

/* ----------------------------------------------------------------- scene */

/* Scene container; replaces Scene (integration/Scene.cu:21-95). */
RT_API int rt_scene_create(rt_context *ctx, rt_scene **out);
RT_API int rt_scene_destroy(rt_scene *scene);

/* Appends a triangle mesh (world-space vertices). Triangles get consecutive global
 * ids in call order — the concatenation order of Scene::build / BVH::initializeTriangles
 * (Scene.cu:64-89, BVH.cu:288-291). `normals`/`nidx` may be NULL (no shading normals);
 * when given, the reference's interpolated shading normal and its 0.15 hit-point
 * offset apply (Triangle.cu:379-419). material: index into the material table.
 * shape_id: the id the reference stores in SurfaceInteraction (meshId, Triangle.cu:427).
 * transparent: 1 when shadow rays ignore these triangles (Triangle.cu:439-440).
 * first_tri (out, nullable): global id of the mesh's first triangle. */
RT_API int rt_scene_add_mesh(rt_scene *scene, const float *xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri,
                      const float *normals, uint32_t nn, const uint32_t *nidx, uint32_t material,
                      int32_t shape_id, int transparent, uint32_t *first_tri);

/* Appends a full sphere of `radius` with the reference's object<->world matrices
 * (row-major 4x4; Sphere(Point3f,Float), shapes/Sphere.cu:233-245). Analytic shapes
 * are reported as prim = RT_PRIM_SHAPE | index. */
RT_API int rt_scene_add_sphere(rt_scene *scene, const float object_to_world[16], const float world_to_object[16],
                        float radius, uint32_t material, int32_t shape_id, int transparent,
                        uint32_t *index);

/* Appends a Plane (shapes/Plane.cu): the unit square [0,1]^2 at z = 0 of its object space, with
 * the reference's object<->world matrices (row-major 4x4: the base change of
 * Plane(bottomLeftCorner, axisX, axisY, normal), Plane.cu:26-50, and its inverse). Its hits are
 * Plane::intersects' arithmetic (Plane.cu:127-170) and are reported as prim = RT_PRIM_SHAPE | index
 * with the object-space (x, y) in the hit's b1, b2; planes and spheres share one index space in
 * the order they were added, as the reference's shape list does (Scene.cu:141-146). */
RT_API int rt_scene_add_plane(rt_scene *scene, const float object_to_world[16], const float world_to_object[16],
                              uint32_t material, int32_t shape_id, int transparent, uint32_t *index);

/* Builds the acceleration structures: the 8-wide compressed BVH used for traversal
 * and the reference-order tree (BVH::BVH, cuda_libraries/BVH.cu:314-341) whose
 * static order breaks exact distance ties like the reference does. Replaces
 * Scene::build (integration/Scene.cu:56-95), whose BVH the reference builds on the host.
 * The 8-wide BVH is a PLOC tree over the reference tree's Morton order, collapsed to 8-wide
 * nodes. Both are built on the GPU unless rt_scene_set_build chose the host. */
RT_API int rt_scene_commit(rt_scene *scene);

#define RT_BUILD_DEVICE 0u /* rt_scene_set_build: build on the GPU (default) */
#define RT_BUILD_HOST 1u   /* build on the host threads; the same bytes as RT_BUILD_DEVICE */
/* Where rt_scene_commit builds. Both produce identical structures. */
RT_API int rt_scene_set_build(rt_scene *scene, uint32_t mode);

/* Copies the committed acceleration structures to host memory, for inspection and
 * serialisation: nodes (80 bytes each), triangle records (48 bytes each: vertices, with
 * the reference traversal rank, the triangle id and the flags in the w lanes) and the
 * reference tree's boxes (6 floats per node, 2n - 1 nodes). Any output may be NULL; a
 * non-NULL one must hold the count the call reports (query the counts with NULL outputs
 * first). */
RT_API int rt_scene_export_bvh(rt_scene *scene, void *nodes, void *records, float *ref_boxes, uint64_t *nnodes,
                               uint64_t *nrecords, uint64_t *nref_nodes);

typedef struct rt_scene_stats {
    uint64_t triangles;
    uint64_t spheres;
    uint64_t bvh8_nodes;
    uint64_t bvh8_leaf_triangles; /* triangle records in BVH8 leaf order */
    uint64_t device_bytes;        /* device memory held by the scene */
    double build_ms;              /* wall time of the last commit (build and upload) */
} rt_scene_stats;
RT_API int rt_scene_stats_get(rt_scene *scene, rt_scene_stats *out);

/* ----------------------------------------------------------------- rays */

#define RT_PRIM_NONE (-1)
#define RT_PRIM_SHAPE ((int32_t)0x40000000) /* analytic shape flag in rt_hit.prim */

/* 32-byte ray: origin + tmax, direction + flags (read as two 16-byte loads). */
typedef struct rt_ray {
    float ox, oy, oz, tmax;
    float dx, dy, dz;
    uint32_t flags; /* reserved, 0 */
} rt_ray;

/* 16-byte hit: distance, primitive (global triangle id, RT_PRIM_SHAPE|shape, or -1),
 * scaled barycentrics b1, b2 of a triangle hit, a plane's object-space (x, y), 0 for spheres. */
typedef struct rt_hit {
    float t;
    int32_t prim;
    float b1, b2;
} rt_hit;

/* Trace flags. */
#define RT_TRACE_SHADOW 0x1u /* checkShadow semantics: skip transparent primitives */
#define RT_TRACE_FAST 0x2u   /* skip the reference-order exactness checks */
#define RT_TRACE_COUNT_ANY 0x4u /* rt_trace_counts: count the any-hit walk instead of the closest-hit one */

/* Closest hit for n rays, device pointers. Replaces BVH::intersectRays
 * (cuda_libraries/BVH.cu:541-584) followed by the analytic-shape loop of
 * Scene::intersects (integration/Scene.cu:108-150): the triangle id equals the one
 * the reference traversal returns (its distance-tie order and its offset-update
 * quirk included), unless RT_TRACE_FAST is given. */
RT_API int rt_trace_closest(rt_scene *scene, const rt_ray *rays_dev, uint64_t n, rt_hit *hits_dev, uint32_t flags);

/* Same with host buffers: copies rays in and hits out inside the call (pinned
 * staging; the end-to-end form the reference's host-vector API corresponds to). */
RT_API int rt_trace_closest_host(rt_scene *scene, const rt_ray *rays, uint64_t n, rt_hit *hits, uint32_t flags);

/* Closest hit exactly like rt_trace_closest, for callers that must not allocate device
 * memory while they trace (a render thread that cannot afford the device synchronisation an
 * allocation may cause, or a host whose own pool allocator owns all device memory). It has
 * no counterpart in the reference. Its scratch (the reference-order replay queue and the
 * counters) is a fixed device array inside this library, about 4 MiB, held on every GPU
 * that loads the library until the process exits. At most 1048576 rays per call
 * (RT_ERR_CAPACITY above that). The first call on a device looks up the array's device
 * address (make that first call before any stream capture) and keeps it for the process's
 * life, so do not call it after a cudaDeviceReset of that device. All calls share the array:
 * calls that overlap on the GPU (other threads or streams) race; serialise them. */
RT_API int rt_trace_closest_noalloc(rt_scene *scene, const rt_ray *rays_dev, uint64_t n, rt_hit *hits_dev,
                                    uint32_t flags);

/* Occlusion test, replacing the shadow-ray use of Scene::intersects in Scene::isVisible
 * (Scene.cu:238-276): rays[i].tmax is the distance to the light. Device pointers.
 * Default: the reference's decision, bit for bit. The ray is traced unbounded (the reference's
 * shadow rays carry tMax = inf) to the closest hit rt_trace_closest reports, and
 * occluded[i] = 1 when there is one at t <= tmax (isVisible: visible = no hit or t > distance).
 * With RT_TRACE_FAST: any-hit traversal that stops at the first primitive hit at t < tmax (the
 * renderer's shadow rays); it can differ from the reference where the reference's offset-update
 * quirk hides an occluder (Triangle.cu:569-593) and at t == tmax.
 * RT_TRACE_SHADOW: transparent primitives do not occlude (checkShadow, Triangle.cu:439-440). */
RT_API int rt_trace_any(rt_scene *scene, const rt_ray *rays_dev, uint64_t n, uint8_t *occluded_dev, uint32_t flags);
/* The same decisions packed into a bit mask: ray i is bit i % 32 of occluded_bits[i / 32]
 * (ceil(n / 32) words, 4-byte aligned; the last word's bits past n are 0). */
RT_API int rt_trace_any_bits(rt_scene *scene, const rt_ray *rays_dev, uint64_t n, uint32_t *occluded_bits_dev,
                             uint32_t flags);

/* Traversal work per ray, the numerator of a traversal roofline (new in this library; the
 * reference has no counterpart). Walks the rays as rt_trace_closest does with RT_TRACE_FAST
 * (or, with RT_TRACE_COUNT_ANY, as rt_trace_any does with RT_TRACE_FAST: the renderer's
 * shadow rays, stopping at the first hit before tmax) and writes, for ray i,
 * counts_dev[2i] = BVH8 nodes visited (80 bytes each) and counts_dev[2i+1] = triangle records
 * tested (48 bytes each). Writes no hits. RT_TRACE_SHADOW: transparent primitives are skipped.
 * counts_dev: 2n uint32, 8-byte aligned. RT_ERR_CAPACITY when a ray's walk ran out of stack
 * (its counts stop there; the other rays' are complete). */
RT_API int rt_trace_counts(rt_scene *scene, const rt_ray *rays_dev, uint64_t n, uint32_t flags, uint32_t *counts_dev);

/* Counters of the last rt_trace_closest call: rays that took the reference-order
 * exact traversal (distance ties resolved through the reference tree, grazing
 * rays, near-zero offsets, and walks deeper than the BVH8 stack, which are replayed
 * there with exact results rather than reported as errors). */
typedef struct rt_trace_stats {
    uint64_t rays;
    uint64_t exact_fallback_rays;
} rt_trace_stats;
RT_API int rt_trace_stats_get(rt_scene *scene, rt_trace_stats *out);


/* ------------------------------------------------------------- materials */

/* Material kinds (materials/*.cu). */
typedef enum rt_material_type {
    RT_MAT_LAMBERTIAN = 0, /* LambertianMaterial / LambertianBRDF (LambertianBSDF.cu:10-77) */
    RT_MAT_TROWBRIDGE = 1, /* TrowbridgeMaterial, GGX conductor (TrowbridgeBSDF.cu:12-253) */
    RT_MAT_DIELECTRIC = 2, /* DielectricMaterial / GlassMaterial (DielectricMaterial.cu:12-83) */
    RT_MAT_LIGHT = 3,      /* LightMaterial: emitter, no scattering (LightMaterial.cu:10-60) */
    RT_MAT_MIRROR = 4,     /* perfect specular reflector (MirrorMaterial.cu) */
    RT_MAT_PLAIN = 5,      /* PlainMaterial: returns its colour on camera hits only */
    RT_MAT_PHONG = 6,      /* PhongMaterial (PhongMaterial.cu): color = kd, k = ks, roughness[0] = ns */
    RT_MAT_SUBSURFACE = 7, /* SSMaterial (SSMaterial.cu): a Phong surface (color = kd, k = ks, roughness[0] = ns)
                              over a medium for the dipole photon estimate: ior = eta, eta = sigma_s,
                              extra = sigma_a, roughness[1] = g (phase asymmetry) */
    RT_MAT_BECKMANN = 8,         /* BeckmannMaterial (BeckmannBSDF.cu): color = kd, eta, k, roughness x/y
                                    (alpha = sqrt(roughness)) */
    RT_MAT_TROWBRIDGE_BASIC = 9, /* TrowbridgeBasicMaterial: RT_MAT_TROWBRIDGE with Fresnel 1 */
    RT_MAT_FRESNEL_BLEND = 10,   /* FresnelBlendMaterial: extra = ke (emission); its constructor fixes
                                    kd = 1, ks = 0 and alpha = 0.5 */
    RT_MAT_PLASTIC = 11,         /* PlasticUnrealMaterial(color, ior): kd = ks = color */
} rt_material_type;

#define RT_MATF_TRANSPARENT 0x1u /* ignored by shadow rays (Material::isTransparent) */

typedef struct rt_material {
    uint32_t type;        /* rt_material_type */
    uint32_t flags;       /* RT_MATF_* */
    float color[3];       /* kd (Lambertian, Trowbridge), ks=kt (Dielectric), emission colour (Light) */
    float intensity;      /* emission scale (Light): Le = color * intensity */
    float eta[3], k[3];   /* conductor Fresnel (Trowbridge) */
    float roughness[2];   /* Trowbridge roughness x/y; alpha = sqrt(roughness) */
    float ior;            /* Dielectric index of refraction (Glass: 1.5) */
    float extra[3];       /* RT_MAT_SUBSURFACE: sigma_a */
    uint32_t texture;     /* 1 + id of a scene texture (rt_scene_add_texture); 0: none. Applied
                             where the reference's materials read their Texture: Lambertian,
                             Phong, Subsurface (surface and dipole kd) and Plain multiply kd by
                             the texel; Trowbridge, TrowbridgeBasic and Beckmann replace kd by
                             it; the other materials ignore it */
} rt_material;

/* A material's BSDF for n direction pairs in the shading frame (normal +z), device arrays of
 * 3 floats per direction: f = what Material::lightReflected returns (f |cos wi| for most
 * materials; Phong and FresnelBlend leave out the cosine, as the reference does) and
 * pdf = Material::pdf (nullable). The renderer's own code (materials/*.cu). Runs on the
 * legacy default stream and returns when done. The directions carry no surface point, so
 * `texture` is not applied: pass the texel-applied kd in `color`. */
RT_API int rt_material_eval(const rt_material *m, const float *wo, const float *wi, uint64_t n, float *f, float *pdf);
/* Material::sampleDirection for n outgoing directions: wi, the value it returns (f |cos| / pdf
 * in the reference's convention), the pdf the renderer pairs with it (nullable) and whether the
 * sample is a delta (nullable, 1 byte each). Sample i uses the random stream (i, seed).
 * flags: RT_RENDER_COMPAT selects the reference's dielectric estimator. */
RT_API int rt_material_sample(const rt_material *m, const float *wo, uint64_t n, uint32_t seed, uint32_t flags, float *wi,
                              float *value, float *pdf, uint8_t *delta);
/* SSMaterial::singleScattering (materials/SSMaterial.cu:108-181) of an RT_MAT_SUBSURFACE
 * material for n cases in the shading frame (device arrays): wo toward the camera, L the light
 * direction (3 floats each), u the sampler's sample in (0, 1) (1 float each). Out: the value (3
 * floats), the refracted light direction Ti and the surface point Pi where the light enters
 * (3 floats each, both nullable). L = 0 gives 0, as the reference's photon case. The reference
 * defines the term but its integrator never calls it; neither does rt_render. */
RT_API int rt_material_single_scattering(const rt_material *m, const float *wo, const float *L, const float *u, uint64_t n,
                                         float *rgb, float *wi, float *point);

/* Replaces the Material* each Shape/Triangle points to (Triangle::setMaterial,
 * Shape::setMaterial): a table indexed by the `material` ids given at add time. */
RT_API int rt_scene_set_materials(rt_scene *scene, const rt_material *table, uint32_t n);

/* Per-triangle material ids for triangles [first, first+n) (overrides the mesh id). */
RT_API int rt_scene_set_triangle_materials(rt_scene *scene, uint32_t first, uint32_t n, const uint32_t *materials);

/* A texture (textures/Texture.cu: Texture::pixelMatrix): width x height RGB texels, 3 floats
 * each, rows in the order Texture::loadBmpImage stores them (row 0 = the BMP's first stored
 * row). Host memory, copied. *id receives the texture's id; materials name it as 1 + id.
 * Takes effect at the next render. */
RT_API int rt_scene_add_texture(rt_scene *scene, const float *rgb, uint32_t width, uint32_t height, uint32_t *id);
/* Texture coordinates of triangles [first, first+n): 6 floats each, the (u, v) of vertices 0,
 * 1 and 2 (TriangleMesh::textureCoords through Triangle::textureIndices). Triangles without
 * them use (0,0), (1,0), (1,1) (Triangle::getSurfaceCoordinates, Triangle.cu:134-151). The
 * hit's surface point is the barycentric blend (Triangle.cu:355-358); a sphere's is its
 * (theta, phi) in degrees (Sphere::localToSurface, Sphere.cu:269-275). */
RT_API int rt_scene_set_triangle_uvs(rt_scene *scene, uint32_t first, uint32_t n, const float *uv);
/* Texture::getColor (Texture.cu:179-192) of texture `id` at n surface points: device arrays,
 * 2 floats in, 3 floats out per point. The texel index is the point times the size, converted
 * to unsigned as the reference's x86-64 build converts it (through a 64-bit integer) and
 * clamped to the last row and column. */
RT_API int rt_texture_lookup(rt_scene *scene, uint32_t id, const float *uv_dev, uint64_t n, float *rgb_dev);

/* PointLight(lightToWorld = translate(pos), color, intensity) (light/PointLight.cu:15-96). */
RT_API int rt_scene_add_point_light(rt_scene *scene, const float pos[3], const float rgb[3], float intensity);

/* ------------------------------------------------------------- rendering */

/* ProjectiveCamera (camera/ProjectiveCamera.cu:10-104): raster -> camera is
 * raster_to_camera (row-major 4x4, projective), camera -> world camera_to_world;
 * lens_radius > 0 enables the thin lens with focal_distance. */
typedef struct rt_camera {
    float camera_to_world[16];
    float raster_to_camera[16];
    float lens_radius;
    float focal_distance;
    uint32_t width, height;
} rt_camera;

#define RT_RENDER_NEE_AREA 0x1u /* next-event estimation on emissive triangles, MIS with BSDF hits */
#define RT_RENDER_COMPAT 0x2u   /* reference estimator quirks (delta-light MIS weight, 0.7/0.3 glass lobes
                                   without pdf, reference Fresnel); off = physically consistent */
#define RT_RENDER_EXACT_TRACE 0x4u /* reference-exact closest-hit ids for extension rays */
#define RT_RENDER_HOST_LOOP 0x80u  /* the host checks for completion after every 4-wave group instead of the
                                      device-side loop (a CUDA graph with a conditional WHILE node); the same
                                      kernels and samples, for tools that do not see kernels inside
                                      conditional graphs */
#define RT_RENDER_STAGE_TIMES 0x100u /* time every wavefront stage with CUDA events (read them with
                                        rt_render_stage_times); implies the host-side loop, launched
                                        without graphs, so it is slower: a profiling aid */
#define RT_RENDER_SUBSURFACE 0x20u /* CHECK_SUBSURFACE_SCATTERING: at camera-ray hits on RT_MAT_SUBSURFACE add
                                      the dipole photon estimate (rt_photon_subsurface, radius 0.3);
                                      needs the photon map of rt_render_set_photon_map */
#define RT_RENDER_HYBRID 0x40u     /* RENDER_MODE HYBRID (Scene.cu:914-969): at every scattering vertex the
                                      direct-light term is (photon density + next-event estimate) / 2 and
                                      the path continues; needs the photon map */
#define RT_RENDER_PHOTON_MAP 0x8u  /* photon-mapping mode (RENDER_MODE PHOTON_MAPPING): at the first
                                      scattering hit the photon density estimate replaces the rest
                                      of the path; needs rt_render_set_photon_map */

typedef struct rt_render_opts {
    uint32_t spp;            /* samples per pixel in this call */
    uint32_t sample_offset;  /* index of the first sample (progressive rendering) */
    uint32_t max_depth;      /* MAX_RAY_RECURSION_DEPTH (types.h:41) */
    uint32_t rr_depth;       /* Russian roulette when depth > rr_depth (pathTracing.cu:91) */
    uint32_t seed;           /* PCG stream base; per-pixel stream = pixel index */
    uint32_t flags;          /* RT_RENDER_* */
    uint32_t max_paths;      /* wavefront capacity (0: automatic) */
    uint32_t reserved;
} rt_render_opts;

typedef struct rt_render_stats {
    uint64_t camera_rays;
    uint64_t extension_rays; /* closest-hit rays incl. camera rays */
    uint64_t shadow_rays;
    uint64_t waves;
    double ms;               /* device time of the render call */
    uint64_t gathers;        /* photon-map estimates (density and dipole) */
} rt_render_stats;

/* Path-traces spp samples per pixel and ADDS them to the caller's film (device
 * buffers, width*height pixels): sum_rgb (3 floats per pixel), count (valid samples
 * per pixel), optional sum_rgb64 (3 doubles per pixel, FP64 accumulation). The pixel
 * estimate is sum/count: samples with NaN/Inf radiance are dropped, which equals the
 * reference's replacement by the mean of the valid ones (pathTracing.cu:457-490).
 * Replaces PathTracerIntegrator::render (integration/PathTracerIntegrator.cu:140-210)
 * with its bounce loop computeSamples (pathTracing.cu:284-414). */
RT_API int rt_render(rt_scene *scene, const rt_camera *camera, const rt_render_opts *opts, float *sum_rgb,
                     uint32_t *count, double *sum_rgb64, rt_render_stats *stats);

/* One view of a batch: the camera and per-view render options of rt_render_opts. */
typedef struct rt_view {
    rt_camera camera;
    uint32_t spp, sample_offset, max_depth, rr_depth, seed;
    uint32_t scene; /* the view's scene in a merged scene (rt_scene_merge: its index in the list); 0 otherwise */
    uint32_t reserved[2];
} rt_view;

/* Many views of one scene in one wavefront (new in this build: the reference renders one
 * camera per PathTracerIntegrator::render call, PathTracerIntegrator.cu:140-210). The views
 * may differ in resolution, spp, depth and seed; their paths share the queues, so small views
 * keep the GPU as busy as one large frame. Films lie back to back: view i's pixels start at
 * pixel sum over k < i of width_k * height_k in sum_rgb (3 floats per pixel), count and sum64
 * (nullable). A view renders exactly the samples rt_render would give it with the same
 * options. flags: RT_RENDER_* for all views; max_paths: queue capacity (0: automatic, the largest
 * power of two up to 2^26 paths whose buffers fit in the smaller of an eighth of the device's
 * memory and a quarter of its free memory, never more paths than the call's samples). */
RT_API int rt_render_batch(rt_scene *scene, const rt_view *views, uint32_t nviews, uint32_t flags, uint32_t max_paths,
                           float *sum_rgb, uint32_t *count, double *sum64, rt_render_stats *stats);

/* Several committed scenes of one context as one scene for rendering (new in this build; the
 * reference renders one scene per PathTracerIntegrator::render call, PathTracerIntegrator.cu:
 * 140-210). rt_render_batch on the result renders views of all of them in one wavefront: a
 * view's `scene` field is the index of its scene in `scenes`, and its paths see only that
 * scene's geometry, materials, textures and lights. Each scene keeps its own BVH (copied, with
 * its indices moved); the sources stay valid and independent. A merged scene is for rendering
 * only: it is not modified, traced with rt_trace_*, or rendered with photon maps or
 * RT_RENDER_EXACT_TRACE (RT_ERR_UNSUPPORTED). At most 256 scenes. Free with rt_scene_destroy. */
RT_API int rt_scene_merge(rt_context *ctx, rt_scene *const *scenes, uint32_t n, rt_scene **out);

/* Material sort of the wavefront (new in this build; the reference shades its samples in pixel
 * order, pathTracing.cu:284-414): before each wave is shaded, every chunk of 2^chunk_log2 queue
 * slots is ordered by the kind of surface its ray hit (a miss, then rt_material_type), so the
 * lanes of a warp mostly run the same BSDF code. chunk_log2 is the sort granularity, 5..13;
 * 0 turns the sort off; a new scene uses 10. Results do not depend on it. Applies to rt_render
 * and rt_render_batch. */
RT_API int rt_render_set_sort(rt_scene *scene, uint32_t chunk_log2);

/* Per-stage device time of the scene's last render call made with RT_RENDER_STAGE_TIMES (new; the
 * reference times whole tiles on the host, PathTracerIntegrator.cu:107-135). ms_out[0..n) gets, in
 * milliseconds summed over the call's waves: 0 closest-hit trace (with its reference-order replay),
 * 1 guide inference, 2 material sort, 3 shading, 4 shadow rays, 5 photon-map gathers, 6 film
 * accumulation. Zeros when the last call did not time its stages. n at most RT_RENDER_STAGES. */
#define RT_RENDER_STAGES 7
RT_API int rt_render_stage_times(rt_scene *scene, double *ms_out, uint32_t n);

/* --------------------------------------------------------------- photons */

typedef struct rt_photon_map rt_photon_map;

/* Photon record, 64 bytes (light/Photon.cu:9-47): where it landed, the direction it
 * arrived along, its power, the shading normal, the shape id of the surface it landed on,
 * and which emitted photon path / bounce produced it. */
typedef struct rt_photon {
    float pos[3];
    int32_t shape_id;
    float dir[3];
    uint32_t path;   /* index of the emitted photon */
    float power[3];
    uint32_t depth;  /* bounce at which it was stored (0 = first hit) */
    float normal[3];
    float reserved;
} rt_photon;

typedef struct rt_photon_trace_stats {
    uint64_t emitted;
    uint64_t stored;
    uint64_t rays;   /* closest-hit rays traced */
    double ms;
} rt_photon_trace_stats;

/* Emits n photons from the scene's point lights — light chosen with probability
 * proportional to its power, direction uniform on the sphere, power I*4pi / n_l / p_l
 * (Scene::generatePhotons, Scene.cu:989-1018; PointLight::sampleLight, PointLight.cu:68-95)
 * — and traces them up to max_depth bounces, storing a photon at every hit on a scattering
 * material with power = carried light * path throughput before that hit's BSDF sample;
 * the path continues by BSDF sampling with Russian roulette after rr_depth (computePhotons /
 * samplePhotonIntersections, integration/photonDispersion.cu:26-172). Photons are ordered
 * by (path, depth), independent of scheduling. flags: RT_RENDER_COMPAT as for rt_render. */
RT_API int rt_photons_trace(rt_scene *scene, uint64_t n, uint32_t max_depth, uint32_t rr_depth, uint32_t seed,
                            uint32_t flags, rt_photon_map **out, rt_photon_trace_stats *stats);

/* A photon map over caller-given points (device pointers: 3 floats per point, optional
 * shape ids) — the same structure rt_photons_trace builds. */
RT_API int rt_photon_map_from_points(rt_context *ctx, const float *pos_dev, const int32_t *shape_dev, uint64_t n,
                                     rt_photon_map **out);

/* Builds the balanced kd-tree (median split on the largest extent, kdtree.h:78-108). */
RT_API int rt_photon_map_build(rt_photon_map *map);

RT_API int rt_photon_map_count(rt_photon_map *map, uint64_t *n);
/* Copies photons [first, first+n) to host memory. */
RT_API int rt_photon_map_get(rt_photon_map *map, uint64_t first, uint64_t n, rt_photon *out_host);
RT_API int rt_photon_map_destroy(rt_photon_map *map);

/* Scene::combinePhotonContributions (Scene.cu:607-635) at nq surface points (device
 * buffers, 3 floats each: position, shading normal, outgoing direction toward the viewer;
 * shape ids nullable): sum over the k nearest photons on the same shape within radius of
 * power * f(wo, -photon direction)|cos| for material `mat`, divided by pi * (largest
 * neighbour distance)^2. out_rgb: 3 floats per point. The points carry no surface
 * coordinates: `mat`'s texture is not applied (give the textured kd in `mat` instead). */
RT_API int rt_photon_density(rt_photon_map *map, const rt_material *mat, const float *points_dev,
                             const float *normals_dev, const float *wo_dev, const int32_t *shape_ids_dev, uint64_t nq,
                             uint32_t k, float radius, float *out_rgb_dev);

/* Scene::combinePhotonsSubsurface (Scene.cu:667-701) at nq points of an RT_MAT_SUBSURFACE
 * material: over all photons within `radius` on the point's shape (0.3 in the reference,
 * Scene.cu:802), sum of power * kd * diffusionTermBSSRDF / (2 pi maxDist^2). wo points to the
 * camera. With no photon in range: NaN with RT_RENDER_COMPAT in flags (the reference's 0 / 0),
 * otherwise 0. Device buffers, out_rgb 3 floats per point. */
RT_API int rt_photon_subsurface(rt_photon_map *map, const rt_material *material, const float *points_dev,
                                const float *normals_dev, const float *wo_dev, const int32_t *shape_ids_dev,
                                uint64_t nq, float radius, uint32_t flags, float *out_rgb_dev);

/* Photon map used by rt_render in RT_RENDER_PHOTON_MAP mode, with the gather size and radius
 * (the reference's MAX_NEIGHBOURS and PHOTON_SEARCH_RADIUS, types.h:57-60). NULL detaches. */
RT_API int rt_render_set_photon_map(rt_scene *scene, rt_photon_map *map, uint32_t k, float radius);

/* k nearest photons per query point within `radius` (distance < radius, same shape id
 * unless the query's id is -1), as nn::KDTree::nearest_neighbors + Scene::search_nearest
 * (kdtree.h:111-197, Scene.cu:704-722). Device pointers: queries 3 floats each,
 * shape_ids (nullable = -1 for all), out_idx nq*k photon indices (-1 padded), out_dist
 * nq*k distances (nullable), out_count nq. Results are ordered by distance. k <= 128. */
RT_API int rt_photon_knn(rt_photon_map *map, const float *queries_dev, const int32_t *shape_ids_dev, uint64_t nq,
                         uint32_t k, float radius, int32_t *out_idx_dev, float *out_dist_dev,
                         uint32_t *out_count_dev);

/* ------------------------------------------------------------ film files and RMSE */

/* Film::storeContributionsToFile (camera/Film.cu:366-391): writes `path`.hdrbmp in the
 * reference's format (text: "P6", resolution, "F", samples per pixel, then per pixel the RGB
 * sum over its samples). The device film is rt_render's: sum_rgb (or sum64 when non-null) and
 * count; a pixel's sum is written as sum * samples / count (NaN/Inf samples replaced by the
 * mean of the valid ones, pathTracing.cu:457-490). */
RT_API int rt_film_store_hdrbmp(const char *path, uint32_t width, uint32_t height, const float *sum_rgb_dev,
                                const uint32_t *count_dev, const double *sum64_dev, uint64_t samples);
/* Film::loadContributionsFromFile (camera/Film.cu:393-449): reads `path`.hdrbmp into host
 * sums (3 doubles per pixel) and its samples per pixel. */
/* Tone mapping of a film to 8-bit RGB (device output, 3 bytes per pixel, film order: the top
 * row first): Film::toneMaxPixel (camera/Film.cu:156-282) with the film's maximum channel
 * and maximum luminance (getMaxChannel / getMaxLuminance, Film.cu:120-153), then
 * (unsigned char)(v * 255) (Film::toneMapBMP / toneMapPPM). The film pixel is the sum over
 * `samples` samples; with `count` (nullable) the sum is first scaled by samples / count, the
 * film rt_film_store_hdrbmp writes. Device pointers; sum_rgb or sum64 (FP64, preferred when
 * given). Runs on the legacy default stream and returns when done. */
#define RT_TONEMAP_EQUALIZE 0u       /* ToneMappingType equalize: p / max */
#define RT_TONEMAP_REINHARD 1u       /* reinhard with the film's maximum luminance */
#define RT_TONEMAP_REINHARD_JODIE 2u /* reinhardJodie */
#define RT_TONEMAP_ACES 3u           /* ACESfilmic */
#define RT_TONEMAP_UNCHARTED2 4u     /* uncharted2 (not clamped, as the reference) */
#define RT_TONEMAP_GAMMA_CLAMP 5u    /* gammaClamp: (p / max)^(1/2.2) */
RT_API int rt_film_tonemap(const float *sum_rgb, const uint32_t *count, const double *sum64, uint64_t npix,
                           uint64_t samples, uint32_t mode, uint8_t *rgb8_dev);
/* 8-bit RGB images (host memory, film order) written as Film::writeToBMP writes them
 * (BitmapImage, camera/BMP_Format.cu: bottom-up BGR rows padded to 4 bytes) and as
 * Film::writeToPPM (camera/Film.cu:339-351). `path` is used as given (the reference appends
 * ".bmp" / ".ppm" to its argument). */
RT_API int rt_image_write_bmp(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height);
RT_API int rt_image_write_ppm(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height);
RT_API int rt_film_load_hdrbmp(const char *path, uint32_t width, uint32_t height, double *sum_rgb_host,
                               uint64_t *samples);
/* computeRMSE (camera/Film.cu:611-632) of two device films on the GPU: sqrt(sum over pixels
 * of |mean_a - mean_b|^2 / pixels), mean = sum / count per pixel (the FP64 sums when given). */
RT_API int rt_film_rmse(const float *sum_a_dev, const uint32_t *count_a_dev, const double *sum64_a_dev,
                        const float *sum_b_dev, const uint32_t *count_b_dev, const double *sum64_b_dev, uint64_t npix,
                        double *rmse);

/* ------------------------------------------------------------ path guide */

/* Learned path-guiding proposal (new in this build; the reference has no counterpart).
 * A small MLP maps an encoded shading point — position (12 frequency bands 2^(k/2) per axis
 * inside the guide's box), outgoing direction (one-blob, 32 theta + 32 phi bins), shading normal:
 * 139 inputs padded to 144 — through 4 hidden layers of 64 (ReLU) to 48 outputs: 8 von
 * Mises-Fisher lobes (mean direction, log concentration, weight logit) and the probability
 * alpha (in [0.05, 0.95]) of sampling the guide rather than the BSDF. FP16 weights and activations on the
 * tensor cores, FP32 accumulation, FP32 master weights with Adam (beta 0.9 / 0.99). */
typedef struct rt_guide rt_guide;

typedef struct rt_guide_opts {
    float bbox_min[3], bbox_max[3]; /* position encoding domain (the scene bounds) */
    float learning_rate;            /* Adam step size; 1e-2 in the guiding configuration */
    uint32_t seed;                  /* weight initialisation */
    uint32_t record_capacity;       /* training records kept per render (0: 4,194,302, the maximum) */
    uint32_t max_depth;             /* vertices at path depth >= max_depth sample the BSDF only (0: no limit) */
} rt_guide_opts;

#define RT_GUIDE_INPUTS 144
#define RT_GUIDE_OUTPUTS 48
#define RT_GUIDE_LOBES 8
#define RT_RENDER_GUIDE 0x10u /* rt_render_opts.flags: sample with the scene's guide (one-sample MIS).
                               * Combines with RT_RENDER_SUBSURFACE and RT_RENDER_HYBRID (their photon
                               * estimates also train the guide); RT_ERR_UNSUPPORTED with
                               * RT_RENDER_PHOTON_MAP, whose paths end where the guide would sample. */

RT_API int rt_guide_create(rt_context *ctx, const rt_guide_opts *opts, rt_guide **out);
RT_API int rt_guide_destroy(rt_guide *g);
/* Parameter count and the FP32 master copy, in this order: for each layer l = 0..4,
 * W_l (inputs x outputs, row-major) then b_l. Setting them resets the Adam moments. */
RT_API int rt_guide_param_count(rt_guide *g, uint64_t *n);
RT_API int rt_guide_params_get(rt_guide *g, float *host, uint64_t n);
RT_API int rt_guide_params_set(rt_guide *g, const float *host, uint64_t n);
RT_API int rt_guide_steps(rt_guide *g, uint64_t *steps); /* Adam steps taken */
/* Back to the freshly created state (seeded weights, zero Adam moments, untrained: renders
 * sample the BSDF until the next training step); device buffers are kept. */
RT_API int rt_guide_reset(rt_guide *g);

/* Raw network outputs for B shading points (device buffers): queries are 9 floats each
 * (position, shading normal, outgoing direction), out is B*48 floats. */
RT_API int rt_guide_eval(rt_guide *g, const float *queries_dev, uint64_t B, float *out_dev);
/* One-sample MIS density alpha * vmf_mixture(dir) + (1 - alpha) * bsdf_pdf at B (query, dir) pairs. */
RT_API int rt_guide_pdf(rt_guide *g, const float *queries_dev, const float *dirs_dev, const float *bsdf_pdf_dev,
                        uint64_t B, float *out_pdf_dev);
/* Direction samples of the vMF mixture alone from 3 uniforms per query; out_pdf: its density there. */
RT_API int rt_guide_sample(rt_guide *g, const float *queries_dev, const float *u3_dev, uint64_t B, float *out_dirs_dev,
                           float *out_pdf_dev);

/* One training step on B samples:
 *   loss = mean_i( -wt_i * log V(dir_i) + wt_i^2 * qc_i / q_i ),
 *   V = the vMF mixture (its KL term fits the lobes), q = alpha * V + (1 - alpha) * bsdf_pdf and
 *   qc = q held constant with V (the estimator's second moment, which trains alpha only),
 *   wt_i = min(w_i / mean(w), 32), w_i = the sample's incident radiance times f * cos / pdf.
 * apply = 0 computes the gradient only; apply = 1 also takes an Adam step. grad_host (nullable)
 * receives the gradient (parameter order as rt_guide_params_get), loss_out (nullable) the loss. */
RT_API int rt_guide_train_step(rt_guide *g, const float *queries_dev, const float *dirs_dev,
                               const float *bsdf_pdf_dev, const float *weights_dev, uint64_t B, int apply,
                               float *grad_host, float *loss_out);

/* Online training on the tracer's own samples. rt_render_set_guide(scene, g, train) makes
 * rt_render with RT_RENDER_GUIDE sample with g; with train != 0 each such call also records
 * every guided vertex (query, sampled direction, BSDF pdf, the radiance the path later
 * carried back through it). rt_guide_train_records then takes `steps` Adam steps on batches
 * of `batch` records drawn (seeded, with replacement) from those with nonzero weight. */
RT_API int rt_render_set_guide(rt_scene *s, rt_guide *g, int train);
RT_API int rt_guide_record_count(rt_guide *g, uint64_t *records, uint64_t *nonzero);
/* Copies records [first, first + n) to host, 20 floats each: position, shading normal, outgoing
 * direction, sampled direction, BSDF pdf of it, throughput before the vertex (rgb), radiance the
 * path carried back through the sampled direction (rgb), previous record of the path (uint32
 * bits; 0x3FFFFF: none). */
RT_API int rt_guide_records_get(rt_guide *g, uint64_t first, uint64_t n, float *host);
RT_API int rt_guide_train_records(rt_guide *g, uint32_t steps, uint32_t batch, uint32_t seed, float *loss_out);

#ifdef __cplusplus
}
#endif
#endif /* RT_B200_H */
