/*
 * Test infrastructure only: plain-C restatement of the reference renderer's
 * closest-hit, sphere and photon-gather arithmetic (hsunekichi/2023_render_engine).
 * See rt_oracle.h. Compiled with -ffp-contract=off and without fast-math so every
 * float operation rounds exactly like the reference's IEEE host build.
 */
#define _GNU_SOURCE
#include "rt_oracle.h"
#include "rt_oracle_internal.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* errorBound(n) = (n*eps)/(1-n*eps) with eps = FLT_EPSILON*0.5 evaluated in double,
 * returned as float (cuda_libraries/math.cu:117-120, types.h:23). */
static float error_bound(int n)
{
    double me = (double)FLT_EPSILON * 0.5;
    return (float)((n * me) / (1 - n * me));
}

struct rto_bvh {
    uint32_t n;
    float *tri;        /* 9 floats per triangle: wp0, wp1, wp2 */
    uint8_t *transparent;
    uint32_t *codes;   /* sorted Morton codes */
    uint32_t *sorted;  /* triangle id at each sorted position (= leaf index) */
    float *boxes;      /* (2n-1) * 6 */
};

/* ------------------------------------------------------------------ build */

/* expandBits / morton3D (cuda_libraries/geometricMath.cu:16-44). The clamps run in
 * double (fmax/fmin), the result is stored back to float before truncation. */
static uint32_t expand_bits(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

static uint32_t morton3d(float x, float y, float z)
{
    x = (float)fmin(fmax((double)x * 1024.0, 0.0), 1023.0);
    y = (float)fmin(fmax((double)y * 1024.0, 0.0), 1023.0);
    z = (float)fmin(fmax((double)z * 1024.0, 0.0), 1023.0);
    return expand_bits((uint32_t)x) * 4 + expand_bits((uint32_t)y) * 2 + expand_bits((uint32_t)z);
}

typedef struct {
    uint32_t code, id;
} key_t_;

static int key_cmp(const void *a, const void *b)
{
    const key_t_ *x = (const key_t_ *)a, *y = (const key_t_ *)b;
    if (x->code != y->code) return x->code < y->code ? -1 : 1;
    if (x->id != y->id) return x->id < y->id ? -1 : 1;
    return 0;
}

int rto_bvh_build(const float *xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri,
                  const uint8_t *transparent, rto_bvh **out)
{
    (void)nv;
    if (ntri < 1) return 1;
    rto_bvh *b = (rto_bvh *)calloc(1, sizeof(rto_bvh));
    b->n = ntri;
    b->tri = (float *)malloc(sizeof(float) * 9 * ntri);
    b->transparent = (uint8_t *)calloc(ntri, 1);
    b->codes = (uint32_t *)malloc(sizeof(uint32_t) * ntri);
    b->sorted = (uint32_t *)malloc(sizeof(uint32_t) * ntri);
    b->boxes = (float *)malloc(sizeof(float) * 6 * (2 * (size_t)ntri - 1));
    for (uint32_t t = 0; t < ntri; t++) {
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) b->tri[9 * t + 3 * k + c] = xyz[3 * idx[3 * t + k] + c];
        if (transparent) b->transparent[t] = transparent[t];
    }
    /* Scene bound: thrust::reduce over Triangle::worldBound with init Bound3f(), whose
     * default is the degenerate box at the origin (Triangle.cu:742-746,
     * geometry/BoundingBox.cu:16-21, :43-48, :102-114). */
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (uint32_t t = 0; t < ntri; t++)
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) {
                float v = b->tri[9 * t + 3 * k + c];
                lo[c] = fminf(lo[c], v);
                hi[c] = fmaxf(hi[c], v);
            }
    float diag[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    key_t_ *keys = (key_t_ *)malloc(sizeof(key_t_) * ntri);
    const float third = (float)1 / 3.0f; /* Point3::operator/ multiplies by 1/f (Point.cu:147-151) */
    for (uint32_t t = 0; t < ntri; t++) {
        const float *p = b->tri + 9 * t;
        float cen[3], u[3];
        for (int c = 0; c < 3; c++) {
            cen[c] = third * ((p[c] + p[3 + c]) + p[6 + c]); /* Triangle::centroid (Triangle.cu:657-664) */
            u[c] = (cen[c] - lo[c]) / diag[c];               /* getUnitCubeCoordinates (BoundingBox.cu:176-183) */
        }
        keys[t].code = morton3d(u[0], u[1], u[2]);
        keys[t].id = t;
    }
    qsort(keys, ntri, sizeof(key_t_), key_cmp); /* thrust::sort on (code, id) tuples */
    for (uint32_t t = 0; t < ntri; t++) {
        b->codes[t] = keys[t].code;
        b->sorted[t] = keys[t].id;
    }
    free(keys);
    /* Leaves 0..n-1 in sorted order (BVH.cu:125-134); node i (i < 2n-2) hangs from
     * n + i/2 as left child when i is even: the FIFO of BVH::generateHierarchy
     * (BVH.cu:153-201) pops after every odd index. Boxes merge bottom-up in index
     * order (BVH.cu:203-212). */
    for (uint32_t i = 0; i < ntri; i++) {
        const float *p = b->tri + 9 * b->sorted[i];
        float *bx = b->boxes + 6 * (size_t)i;
        for (int c = 0; c < 3; c++) {
            /* Bound3f(p0, p1) + p2 (Triangle.cu:123-131) */
            float mn = fminf(p[c], p[3 + c]), mx = fmaxf(p[c], p[3 + c]);
            bx[c] = fminf(mn, p[6 + c]);
            bx[3 + c] = fmaxf(mx, p[6 + c]);
        }
    }
    for (size_t i = ntri; i + 1 < 2 * (size_t)ntri; i++) {
        size_t l = 2 * (i - ntri), r = l + 1;
        float *bx = b->boxes + 6 * i;
        const float *bl = b->boxes + 6 * l, *br = b->boxes + 6 * r;
        for (int c = 0; c < 3; c++) {
            bx[c] = fminf(bl[c], br[c]);
            bx[3 + c] = fmaxf(bl[3 + c], br[3 + c]);
        }
    }
    *out = b;
    return 0;
}

void rto_bvh_free(rto_bvh *b)
{
    if (!b) return;
    free(b->tri);
    free(b->transparent);
    free(b->codes);
    free(b->sorted);
    free(b->boxes);
    free(b);
}

void rto_bvh_export(const rto_bvh *b, float *boxes, uint32_t *codes, uint32_t *sorted)
{
    if (boxes) memcpy(boxes, b->boxes, sizeof(float) * 6 * (2 * (size_t)b->n - 1));
    if (codes) memcpy(codes, b->codes, sizeof(uint32_t) * b->n);
    if (sorted) memcpy(sorted, b->sorted, sizeof(uint32_t) * b->n);
}

/* Static traversal order of BVH::intersectRay (BVH.cu:392-445) when every box is hit:
 * at a node's pop its leaf children are tested left then right; interior children
 * are pushed left then right, so the right subtree runs before the left one. */
void rto_bvh_tie_rank(const rto_bvh *b, uint32_t *rank)
{
    uint32_t n = b->n;
    if (n == 1) {
        rank[b->sorted[0]] = 0;
        return;
    }
    uint32_t *stack = (uint32_t *)malloc(sizeof(uint32_t) * 2 * n);
    int sp = 0;
    uint32_t next = 0;
    stack[sp++] = 2 * n - 2;
    while (sp > 0) {
        uint32_t node = stack[--sp];
        uint32_t ch[2] = {2 * (node - n), 2 * (node - n) + 1};
        for (int k = 0; k < 2; k++) {
            if (ch[k] < n)
                rank[b->sorted[ch[k]]] = next++;
            else
                stack[sp++] = ch[k];
        }
    }
    free(stack);
}

/* ------------------------------------------------------------ intersection */

/* Bound3f::intersects (geometry/BoundingBox.cu:296-329): slab test with the ray's
 * invDirection; min/max are fminf/fmaxf (the CUDA host overloads). */
static int box_intersects(const float *bx, const float *o, const float *inv, float tmax)
{
    float tx1 = (bx[0] - o[0]) * inv[0];
    float tx2 = (bx[3] - o[0]) * inv[0];
    float tmin = fminf(tx1, tx2);
    float tmx = fmaxf(tx1, tx2);
    float ty1 = (bx[1] - o[1]) * inv[1];
    float ty2 = (bx[4] - o[1]) * inv[1];
    tmin = fmaxf(tmin, fminf(ty1, ty2));
    tmx = fminf(tmx, fmaxf(ty1, ty2));
    float tz1 = (bx[2] - o[2]) * inv[2];
    float tz2 = (bx[5] - o[2]) * inv[2];
    tmin = fmaxf(tmin, fminf(tz1, tz2));
    tmx = fminf(tmx, fmaxf(tz1, tz2));
    float h = (tmin > 0) ? tmin : tmx;
    return tmx >= tmin && h >= 0 && h <= tmax;
}

/* The geometric part of Triangle::intersects (Triangle.cu:442-593). Returns 0 when
 * the triangle is missed; otherwise the hit offset and its error bound deltaT. */
static int tri_geom_b(const float *v, const float *o, const float *d, float tmax, float *tOut, float *dtOut,
                      float *b1Out, float *b2Out)
{
    float lp0[3], lp1[3], lp2[3];
    for (int c = 0; c < 3; c++) {
        lp0[c] = v[c] - o[c];
        lp1[c] = v[3 + c] - o[c];
        lp2[c] = v[6 + c] - o[c];
    }
    float ad[3] = {fabsf(d[0]), fabsf(d[1]), fabsf(d[2])};
    int kz = (ad[0] > ad[1]) ? 0 : 1;
    if (ad[2] > ad[kz]) kz = 2;
    int kx = kz + 1;
    if (kx == 3) kx = 0;
    int ky = kx + 1;
    if (ky == 3) ky = 0;
    float dx = d[kx], dy = d[ky], dz = d[kz];
    float p0x = lp0[kx], p0y = lp0[ky], p0z = lp0[kz];
    float p1x = lp1[kx], p1y = lp1[ky], p1z = lp1[kz];
    float p2x = lp2[kx], p2y = lp2[ky], p2z = lp2[kz];
    float Sx = -dx / dz;
    float Sy = -dy / dz;
    float Sz = 1.f / dz;
    p0x += Sx * p0z;
    p0y += Sy * p0z;
    p1x += Sx * p1z;
    p1y += Sy * p1z;
    p2x += Sx * p2z;
    p2y += Sy * p2z;
    float e0 = p1x * p2y - p1y * p2x;
    float e1 = p2x * p0y - p2y * p0x;
    float e2 = p0x * p1y - p0y * p1x;
    if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
        /* double-precision recomputation (Triangle.cu:507-522) */
        double a = (double)p2x * (double)p1y;
        double bb = (double)p2y * (double)p1x;
        e0 = (float)(bb - a);
        a = (double)p0x * (double)p2y;
        bb = (double)p0y * (double)p2x;
        e1 = (float)(bb - a);
        a = (double)p1x * (double)p0y;
        bb = (double)p1y * (double)p0x;
        e2 = (float)(bb - a);
    }
    if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return 0;
    float det = e0 + e1 + e2;
    if (det == 0) return 0;
    p0z *= Sz;
    p1z *= Sz;
    p2z *= Sz;
    float so = e0 * p0z + e1 * p1z + e2 * p2z;
    if (det < 0 && (so >= 0 || so < tmax * det)) return 0;
    if (det > 0 && (so <= 0 || so > tmax * det)) return 0;
    float invDet = 1 / det;
    float t = so * invDet;
    float maxZt = fmaxf(fabsf(p0z), fmaxf(fabsf(p1z), fabsf(p2z)));
    float deltaZ = error_bound(3) * maxZt;
    float maxXt = fmaxf(fabsf(p0x), fmaxf(fabsf(p1x), fabsf(p2x)));
    float maxYt = fmaxf(fabsf(p0y), fmaxf(fabsf(p1y), fabsf(p2y)));
    float deltaX = error_bound(5) * (maxXt + maxZt);
    float deltaY = error_bound(5) * (maxYt + maxZt);
    float deltaE = 2 * (error_bound(2) * maxXt * maxYt + deltaY * maxXt + deltaX * maxYt);
    float maxE = fmaxf(fabsf(e0), fmaxf(fabsf(e1), fabsf(e2)));
    float deltaT = 3 * (error_bound(3) * maxE * maxZt + deltaE * maxZt + deltaZ * maxE) * fabsf(invDet);
    *tOut = t;
    *dtOut = deltaT;
    if (b1Out) *b1Out = e1 * invDet;
    if (b2Out) *b2Out = e2 * invDet;
    return 1;
}

static int tri_geom(const float *v, const float *o, const float *d, float tmax, float *tOut, float *dtOut)
{
    return tri_geom_b(v, o, d, tmax, tOut, dtOut, NULL, NULL);
}

/* Triangle::intersects with the reference's running-offset semantics
 * (Triangle.cu:569-593: the offset is lowered before the error-bound rejection). */
static int tri_intersects_seq(const rto_bvh *b, uint32_t tri, const float *o, const float *d, float tmax,
                              float *h, int checkShadow)
{
    if (checkShadow && b->transparent[tri]) return 0;
    float t, dt;
    if (!tri_geom(b->tri + 9 * (size_t)tri, o, d, tmax, &t, &dt)) return 0;
    if (t > *h) return 0;
    *h = t;
    if (*h <= dt) return 0;
    return 1;
}

int rto_triangle_intersects(const rto_bvh *b, uint32_t tri, const float *o, const float *d, float tmax,
                            float *hitOffset, int checkShadow)
{
    return tri_intersects_seq(b, tri, o, d, tmax, hitOffset, checkShadow);
}

static int32_t trace_one(const rto_bvh *b, const float *o, const float *d, float tmax, int checkShadow,
                         float *tOut)
{
    float inv[3] = {1 / d[0], 1 / d[1], 1 / d[2]}; /* Ray ctor (geometry/Ray.cu:32-39) */
    float h = INFINITY;
    int32_t hit = -1;
    uint32_t n = b->n;
    if (n == 1) {
        if (tri_intersects_seq(b, b->sorted[0], o, d, tmax, &h, checkShadow)) hit = (int32_t)b->sorted[0];
        *tOut = h;
        return hit;
    }
    uint32_t stack[64];
    int sp = 0;
    stack[sp++] = 2 * n - 2;
    while (sp > 0) {
        uint32_t node = stack[--sp];
        uint32_t ch[2] = {2 * (node - n), 2 * (node - n) + 1};
        for (int k = 0; k < 2; k++) {
            uint32_t c = ch[k];
            if (c < n) {
                uint32_t tri = b->sorted[c];
                if (tri_intersects_seq(b, tri, o, d, tmax, &h, checkShadow)) hit = (int32_t)tri;
            } else if (box_intersects(b->boxes + 6 * (size_t)c, o, inv, tmax)) {
                if (sp < 64) stack[sp++] = c;
            }
        }
    }
    *tOut = h;
    return hit;
}

void rto_trace_one_full(const rto_bvh *b, const float *o, const float *d, float tmax, int checkShadow,
                        int32_t *id, float *t, float *b1, float *b2)
{
    float tt;
    int32_t h = trace_one(b, o, d, tmax, checkShadow, &tt);
    *id = h;
    *t = tt;
    *b1 = *b2 = 0.f;
    if (h >= 0) {
        float t2, dt;
        tri_geom_b(b->tri + 9 * (size_t)h, o, d, tmax, &t2, &dt, b1, b2);
    }
}

void rto_triangle_vertices(const rto_bvh *b, uint32_t tri, float *v9)
{
    memcpy(v9, b->tri + 9 * (size_t)tri, 9 * sizeof(float));
}

uint32_t rto_bvh_ntri(const rto_bvh *b) { return b->n; }

/* -------------------------------------------------------------- threading */

typedef struct {
    uint64_t n;
    int nthreads;
    void (*fn)(void *ctx, uint64_t i);
    void *ctx;
    uint64_t next;
    pthread_mutex_t mu;
} pool_t;

static void *pool_worker(void *arg)
{
    pool_t *p = (pool_t *)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        uint64_t b = p->next;
        p->next += 1024;
        pthread_mutex_unlock(&p->mu);
        if (b >= p->n) break;
        uint64_t e = b + 1024 < p->n ? b + 1024 : p->n;
        for (uint64_t i = b; i < e; i++) p->fn(p->ctx, i);
    }
    return NULL;
}

static void parallel_for(uint64_t n, int nthreads, void (*fn)(void *, uint64_t), void *ctx)
{
    if (nthreads <= 1 || n < 2048) {
        for (uint64_t i = 0; i < n; i++) fn(ctx, i);
        return;
    }
    pool_t p;
    p.n = n;
    p.nthreads = nthreads;
    p.fn = fn;
    p.ctx = ctx;
    p.next = 0;
    pthread_mutex_init(&p.mu, NULL);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, pool_worker, &p);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&p.mu);
}

typedef struct {
    const rto_bvh *b;
    const float *o, *d, *tmax;
    int checkShadow;
    int32_t *out;
    float *tOut;
} trace_ctx;

static void trace_fn(void *c, uint64_t i)
{
    trace_ctx *t = (trace_ctx *)c;
    float tt;
    int32_t h = trace_one(t->b, t->o + 3 * i, t->d + 3 * i, t->tmax ? t->tmax[i] : INFINITY, t->checkShadow, &tt);
    t->out[i] = h;
    if (t->tOut) t->tOut[i] = h >= 0 ? tt : INFINITY;
}

void rto_trace_ref_order(const rto_bvh *b, const float *o, const float *d, const float *tmax, uint64_t n,
                         int checkShadow, int32_t *out, float *tOut, int nthreads)
{
    trace_ctx c = {b, o, d, tmax, checkShadow, out, tOut};
    parallel_for(n, nthreads, trace_fn, &c);
}

/* ----------------------------------------------------------------- sphere */

typedef struct {
    float v, e;
} ef_t; /* ErrorFloat (cuda_libraries/types.h:92-220) */

static ef_t ef(float v, float e)
{
    ef_t r = {v, e};
    return r;
}
static ef_t ef_add(ef_t a, ef_t b) { return ef(a.v + b.v, a.e + b.e); }
static ef_t ef_sub(ef_t a, ef_t b) { return ef(a.v - b.v, a.e + b.e); }
static ef_t ef_mul(ef_t a, ef_t b)
{
    ef_t r;
    r.v = a.v * b.v;
    r.e = fabsf(r.v) * b.e + fabsf(b.v) * a.e;
    return r;
}
static ef_t ef_smul(float s, ef_t b) /* operator*(Float, ErrorFloat) (types.h:204-211) */
{
    ef_t r;
    r.v = s * b.v;
    r.e = fabsf(r.v) * b.e;
    return r;
}
static ef_t ef_div(ef_t a, ef_t b)
{
    ef_t r;
    r.v = a.v / b.v;
    r.e = (fabsf(r.v) * b.e + fabsf(b.v) * a.e) / (b.v * b.v);
    return r;
}
static ef_t ef_sqrt(ef_t f) /* sqrt(ErrorFloat) (types.h:213-220): the error term runs in double */
{
    ef_t r;
    r.v = sqrtf(f.v);
    r.e = (float)(0.5 * (double)f.e / (double)r.v);
    return r;
}

int rto_sphere_intersects(const float *m, float radius, const float *o, const float *d, float tmax,
                          float *hitOffset)
{
    /* Transform::operator()(Ray, oErr, dErr) const (transformations/Transform.cu:387-404)
     * with the const point/vector overloads (Transform.cu:328-372). */
    const float eb3 = error_bound(3);
    float oe[3], de[3], po[3], pd[3];
    for (int r = 0; r < 3; r++) {
        const float *row = m + 4 * r;
        oe[r] = (fabsf(row[0] * o[0]) + fabsf(row[1] * o[1]) + fabsf(row[2] * o[2]) + fabsf(row[3])) * eb3;
        de[r] = (fabsf(row[0] * d[0]) + fabsf(row[1] * d[1]) + fabsf(row[2] * d[2])) * eb3;
        po[r] = row[0] * o[0] + row[1] * o[1] + row[2] * o[2] + row[3];
        pd[r] = row[0] * d[0] + row[1] * d[1] + row[2] * d[2];
    }
    float wp = m[12] * o[0] + m[13] * o[1] + m[14] * o[2] + m[15];
    float invw = (float)1 / wp;
    for (int r = 0; r < 3; r++) po[r] = invw * po[r];
    float ls = pd[0] * pd[0] + pd[1] * pd[1] + pd[2] * pd[2];
    float tm = tmax;
    if (ls > 0) {
        float dt = (fabsf(pd[0]) * oe[0] + fabsf(pd[1]) * oe[1] + fabsf(pd[2]) * oe[2]) / ls;
        for (int r = 0; r < 3; r++) po[r] = po[r] + pd[r] * dt;
        tm = tm - dt;
    }
    /* normalize (geometry/Vector.cu:454-456, :171-177) */
    float len = sqrtf(pd[0] * pd[0] + pd[1] * pd[1] + pd[2] * pd[2]);
    float il = (float)1 / len;
    for (int r = 0; r < 3; r++) pd[r] = pd[r] * il;
    /* getSphereCollisions (Sphere.cu:18-39) */
    ef_t ox = ef(po[0], oe[0]), oy = ef(po[1], oe[1]), oz = ef(po[2], oe[2]);
    ef_t dx = ef(pd[0], de[0]), dy = ef(pd[1], de[1]), dz = ef(pd[2], de[2]);
    ef_t a = ef_add(ef_add(ef_mul(dx, dx), ef_mul(dy, dy)), ef_mul(dz, dz));
    ef_t b = ef_smul(2.0f, ef_add(ef_add(ef_mul(dx, ox), ef_mul(dy, oy)), ef_mul(dz, oz)));
    ef_t c = ef_sub(ef_add(ef_add(ef_mul(ox, ox), ef_mul(oy, oy)), ef_mul(oz, oz)),
                    ef_mul(ef(radius, 0), ef(radius, 0)));
    /* quadratic (cuda_libraries/math.cu:91-115) */
    ef_t disc = ef_sub(ef_mul(b, b), ef_mul(ef_smul(4.0f, a), c));
    if (disc.v < 0.0f) return 0;
    ef_t rd = ef_sqrt(disc);
    ef_t q = (b.v < 0.0f) ? ef_smul(-0.5f, ef_sub(b, rd)) : ef_smul(-0.5f, ef_add(b, rd));
    ef_t t0 = ef_div(q, a), t1 = ef_div(c, q);
    if (t0.v > t1.v) {
        ef_t tmp = t0;
        t0 = t1;
        t1 = tmp;
    }
    if (t0.v != t0.v || t0.e != t0.e || t1.v != t1.v || t1.e != t1.e) return 0;
    /* checkRayBounds (Sphere.cu:41-81); the full sphere never clips (Sphere.cu:83-124). */
    if (t0.v + t0.e > tm || t1.v - t1.e <= 0) return 0;
    ef_t th = t0;
    if (t0.v - t0.e <= 0) {
        th = t1;
        if (t1.v + t1.e > tm) return 0;
    }
    if (th.v < *hitOffset) { /* Sphere.cu:390-397 */
        *hitOffset = th.v;
        return 1;
    }
    return 0;
}

/* ------------------------------------------------------------------- kNN */

typedef struct {
    const float *pos;
    const int32_t *shape;
    uint64_t n;
    const float *q;
    const int32_t *qshape;
    uint32_t k;
    float radius;
    int32_t *outIdx;
    float *outDist;
    uint32_t *outCount;
} knn_ctx;

/* Euclidean norm as the reference computes it: s = 0; s += r*r per axis; sqrt
 * (kdtree.h:175-176), with r = query - photon per axis (kdtree.h:67-76). */
static float knn_dist(const float *p, const float *q)
{
    float s = 0;
    for (int c = 0; c < 3; c++) {
        float r = q[c] - p[c];
        s += r * r;
    }
    return sqrtf(s);
}

static void knn_fn(void *cv, uint64_t i)
{
    knn_ctx *c = (knn_ctx *)cv;
    const float *q = c->q + 3 * i;
    int32_t sid = c->qshape ? c->qshape[i] : -1;
    uint32_t k = c->k;
    int32_t *bi = c->outIdx + i * k;
    float *bd = c->outDist + i * k;
    uint32_t cnt = 0;
    for (uint64_t j = 0; j < c->n; j++) {
        if (sid != -1 && c->shape[j] != sid) continue;
        float dd = knn_dist(c->pos + 3 * j, q);
        if (!(dd < c->radius)) continue;
        if (cnt == k && !(dd < bd[k - 1])) continue;
        uint32_t p = cnt < k ? cnt++ : k - 1;
        while (p > 0 && (bd[p - 1] > dd)) {
            bd[p] = bd[p - 1];
            bi[p] = bi[p - 1];
            p--;
        }
        bd[p] = dd;
        bi[p] = (int32_t)j;
    }
    for (uint32_t j = cnt; j < k; j++) {
        bi[j] = -1;
        bd[j] = INFINITY;
    }
    c->outCount[i] = cnt;
}

void rto_knn_brute(const float *pos, const int32_t *shape, uint64_t n, const float *q, const int32_t *qshape,
                   uint64_t nq, uint32_t k, float radius, int32_t *outIdx, float *outDist, uint32_t *outCount,
                   int nthreads)
{
    knn_ctx c = {pos, shape, n, q, qshape, k, radius, outIdx, outDist, outCount};
    if (k == 0) {
        for (uint64_t i = 0; i < nq; i++) outCount[i] = 0;
        return;
    }
    parallel_for(nq, nthreads, knn_fn, &c);
}
