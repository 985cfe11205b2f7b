/*
 * Test infrastructure only (the checker, never the product): a plain-C restatement
 * of the reference renderer's hot-path arithmetic, hsunekichi/2023_render_engine.
 * Each function cites the reference file:line it restates. Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load the library built from rt_oracle.c.
 *
 * Parity pin: tests/test_oracle_pin.py checks every function here against the
 * reference's own code compiled from its sources (oracle/ref_harness.cu), and
 * tests/golden/ holds fixtures generated by that reference build.
 */
#ifndef RT_ORACLE_H
#define RT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rto_bvh rto_bvh;

/* Reference BVH (cuda_libraries/BVH.cu:314-341): Morton sort + FIFO pairing tree. */
int rto_bvh_build(const float *xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri,
                  const uint8_t *transparent, rto_bvh **out);
void rto_bvh_free(rto_bvh *b);
/* boxes: (2N-1)*6 floats (pMin, pMax); codes/sorted: N each. */
void rto_bvh_export(const rto_bvh *b, float *boxes, uint32_t *codes, uint32_t *sorted);
/* Position of each triangle in the static reference traversal order (tie rank). */
void rto_bvh_tie_rank(const rto_bvh *b, uint32_t *rank);

/* BVH::intersectRay (BVH.cu:355-448), sequential semantics, nthreads host threads. */
void rto_trace_ref_order(const rto_bvh *b, const float *o, const float *d, const float *tmax,
                         uint64_t n, int checkShadow, int32_t *out, float *tOut, int nthreads);

/* Triangle::intersects (Triangle.cu:434-643) on triangle `tri`; updates *hitOffset. */
int rto_triangle_intersects(const rto_bvh *b, uint32_t tri, const float *o, const float *d,
                            float tmax, float *hitOffset, int checkShadow);

/* Sphere::intersects (Sphere.cu:357-398) given the sphere's worldToObject matrix
 * (row-major 4x4) and radius; returns 1 and the hit offset when it hits. */
int rto_sphere_intersects(const float *w2o, float radius, const float *o, const float *d,
                          float tmax, float *hitOffset);

/* k nearest photons (kdtree.h:111-152 semantics: same shape id unless shape==-1,
 * distance < radius, the k smallest distances) by brute force. Indices sorted by
 * (distance, index); count per query. */
void rto_knn_brute(const float *pos, const int32_t *shape, uint64_t n, const float *q,
                   const int32_t *qshape, uint64_t nq, uint32_t k, float radius,
                   int32_t *outIdx, float *outDist, uint32_t *outCount, int nthreads);

/* ---- path tracing estimator (pt_oracle.c) ---- */

typedef struct pto_material { /* same layout as rt_material in include/rt_b200.h */
    uint32_t type, flags;
    float color[3];
    float intensity;
    float eta[3], k[3];
    float roughness[2];
    float ior;
    float extra[3];
    uint32_t texture; /* not restated here: texture parity is checked against the reference's Texture */
} pto_material;

typedef struct pto_sphere {
    float w2o[16];
    float o2w[16];
    float radius;
    uint32_t material;
} pto_sphere;

typedef struct pto_camera { /* same layout as rt_camera */
    float camera_to_world[16];
    float raster_to_camera[16];
    float lens_radius, focal_distance;
    uint32_t width, height;
} pto_camera;

/* Renders pixels [pix_begin, pix_end) with spp samples each into sum (3 doubles per
 * pixel, indexed by pixel) and count; flags: 1 = area-light NEE, 2 = reference quirks. */
/* The estimator's Phong BSDF (f * |cos|, pdf) for n shading-space pairs (tests). */
void pto_phong_eval(const pto_material *m, const float *wo, const float *wi, uint32_t n, float *out_f, float *out_pdf);

int pto_render(const rto_bvh *bvh, const uint32_t *tri_mat, const pto_sphere *sph, uint32_t nsph,
               const pto_material *mats, uint32_t nmat, const float *plights, uint32_t npl, const pto_camera *cam,
               uint32_t spp, uint32_t sample_offset, uint32_t max_depth, uint32_t rr_depth, uint32_t seed,
               uint32_t flags, uint32_t pix_begin, uint32_t pix_end, double *sum, uint32_t *count, int nthreads);

/* Photon tracing restated (pt_oracle.c): returns the number of photons stored (written up
 * to cap, 16 floats each in rt_photon layout) in (path, depth) order. plights: 6 floats per
 * light (position, rgb*intensity); plight_rgbi: 4 floats per light (rgb, intensity). */
uint64_t pto_trace_photons(const rto_bvh *bvh, const uint32_t *tri_mat, const int32_t *tri_shape,
                           const pto_sphere *sph, const int32_t *sph_shape, uint32_t nsph, const pto_material *mats,
                           uint32_t nmat, const float *plights, const float *plight_rgbi, uint32_t npl, uint64_t n,
                           uint32_t max_depth, uint32_t rr_depth, uint32_t seed, uint32_t flags, float *out,
                           uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif
