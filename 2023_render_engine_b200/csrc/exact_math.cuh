// Device arithmetic that rounds exactly like the reference renderer's IEEE host build.
// Every product and sum goes through the _rn intrinsics, which the compiler never
// contracts into FMAs, and every division is the IEEE one.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rtb {

// errorBound(n) = (n*eps)/(1-n*eps), eps = FLT_EPSILON*0.5, evaluated in double and
// returned as float (cuda_libraries/math.cu:117-120, types.h:23).
constexpr double kMachEps = 5.9604644775390625e-08;  // 2^-24
__host__ __device__ constexpr float error_bound(int n) { return (float)((n * kMachEps) / (1 - n * kMachEps)); }

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ float sel3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

// Per-ray part of the watertight test (Triangle.cu:456-495): axis permutation by the
// largest |direction| component and the shear coefficients. The reference recomputes
// these per triangle; they depend on the ray only.
struct WatertightRay {
    float ox, oy, oz;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    float tmax;
};

__device__ __forceinline__ WatertightRay make_watertight(float ox, float oy, float oz, float dx, float dy, float dz,
                                                         float tmax)
{
    WatertightRay w;
    w.ox = ox;
    w.oy = oy;
    w.oz = oz;
    w.tmax = tmax;
    float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    int kz = (ax > ay) ? 0 : 1;
    float akz = kz == 0 ? ax : ay;
    if (az > akz) kz = 2;
    int kx = kz + 1;
    if (kx == 3) kx = 0;
    int ky = kx + 1;
    if (ky == 3) ky = 0;
    w.kx = kx;
    w.ky = ky;
    w.kz = kz;
    float pdx = sel3(dx, dy, dz, kx), pdy = sel3(dx, dy, dz, ky), pdz = sel3(dx, dy, dz, kz);
    w.Sx = fdiv(-pdx, pdz);
    w.Sy = fdiv(-pdy, pdz);
    w.Sz = fdiv(1.f, pdz);
    return w;
}

struct TriHit {
    float t;       // hit offset
    float e0, e1, e2, invDet;
    float p0z, p1z, p2z, maxXt, maxYt;  // kept for the error bound
};

// Geometric part of Triangle::intersects (Triangle.cu:442-573): returns false when the
// ray misses; otherwise the offset t and what the error bound needs.
__device__ __forceinline__ bool watertight_test(const WatertightRay &w, float4 a, float4 b, float4 c, TriHit &h)
{
    float l0x = fsub(a.x, w.ox), l0y = fsub(a.y, w.oy), l0z = fsub(a.z, w.oz);
    float l1x = fsub(b.x, w.ox), l1y = fsub(b.y, w.oy), l1z = fsub(b.z, w.oz);
    float l2x = fsub(c.x, w.ox), l2y = fsub(c.y, w.oy), l2z = fsub(c.z, w.oz);
    float p0x = sel3(l0x, l0y, l0z, w.kx), p0y = sel3(l0x, l0y, l0z, w.ky), p0z = sel3(l0x, l0y, l0z, w.kz);
    float p1x = sel3(l1x, l1y, l1z, w.kx), p1y = sel3(l1x, l1y, l1z, w.ky), p1z = sel3(l1x, l1y, l1z, w.kz);
    float p2x = sel3(l2x, l2y, l2z, w.kx), p2y = sel3(l2x, l2y, l2z, w.ky), p2z = sel3(l2x, l2y, l2z, w.kz);
    p0x = fadd(p0x, fmul(w.Sx, p0z));
    p0y = fadd(p0y, fmul(w.Sy, p0z));
    p1x = fadd(p1x, fmul(w.Sx, p1z));
    p1y = fadd(p1y, fmul(w.Sy, p1z));
    p2x = fadd(p2x, fmul(w.Sx, p2z));
    p2y = fadd(p2y, fmul(w.Sy, p2z));
    float e0 = fsub(fmul(p1x, p2y), fmul(p1y, p2x));
    float e1 = fsub(fmul(p2x, p0y), fmul(p2y, p0x));
    float e2 = fsub(fmul(p0x, p1y), fmul(p0y, p1x));
    if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
        // double-precision recomputation (Triangle.cu:507-522)
        e0 = __double2float_rn(__dsub_rn(__dmul_rn((double)p2y, (double)p1x), __dmul_rn((double)p2x, (double)p1y)));
        e1 = __double2float_rn(__dsub_rn(__dmul_rn((double)p0y, (double)p2x), __dmul_rn((double)p0x, (double)p2y)));
        e2 = __double2float_rn(__dsub_rn(__dmul_rn((double)p1y, (double)p0x), __dmul_rn((double)p1x, (double)p0y)));
    }
    if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return false;
    float det = fadd(fadd(e0, e1), e2);
    if (det == 0) return false;
    p0z = fmul(p0z, w.Sz);
    p1z = fmul(p1z, w.Sz);
    p2z = fmul(p2z, w.Sz);
    float so = fadd(fadd(fmul(e0, p0z), fmul(e1, p1z)), fmul(e2, p2z));
    float lim = fmul(w.tmax, det);
    if (det < 0 && (so >= 0 || so < lim)) return false;
    if (det > 0 && (so <= 0 || so > lim)) return false;
    float invDet = fdiv(1.0f, det);
    h.t = fmul(so, invDet);
    h.e0 = e0;
    h.e1 = e1;
    h.e2 = e2;
    h.invDet = invDet;
    h.p0z = p0z;
    h.p1z = p1z;
    h.p2z = p2z;
    h.maxXt = fmaxf(fabsf(p0x), fmaxf(fabsf(p1x), fabsf(p2x)));
    h.maxYt = fmaxf(fabsf(p0y), fmaxf(fabsf(p1y), fabsf(p2y)));
    return true;
}

// The conservative error bound of the hit offset (Triangle.cu:575-589).
__device__ __forceinline__ float watertight_delta_t(const TriHit &h)
{
    const float eb2 = error_bound(2), eb3 = error_bound(3), eb5 = error_bound(5);
    float maxZt = fmaxf(fabsf(h.p0z), fmaxf(fabsf(h.p1z), fabsf(h.p2z)));
    float deltaZ = fmul(eb3, maxZt);
    float deltaX = fmul(eb5, fadd(h.maxXt, maxZt));
    float deltaY = fmul(eb5, fadd(h.maxYt, maxZt));
    float deltaE =
        fmul(2.0f, fadd(fadd(fmul(fmul(eb2, h.maxXt), h.maxYt), fmul(deltaY, h.maxXt)), fmul(deltaX, h.maxYt)));
    float maxE = fmaxf(fabsf(h.e0), fmaxf(fabsf(h.e1), fabsf(h.e2)));
    float s = fadd(fadd(fmul(fmul(eb3, maxE), maxZt), fmul(deltaE, maxZt)), fmul(deltaZ, maxE));
    return fmul(fmul(3.0f, s), fabsf(h.invDet));
}

// Bound3f::intersects (geometry/BoundingBox.cu:296-329) with the ray's invDirection.
__device__ __forceinline__ bool ref_box_test(float lx, float ly, float lz, float hx, float hy, float hz, float ox,
                                             float oy, float oz, float ix, float iy, float iz, float tmax)
{
    float tx1 = fmul(fsub(lx, ox), ix), tx2 = fmul(fsub(hx, ox), ix);
    float tmin = fminf(tx1, tx2), tmx = fmaxf(tx1, tx2);
    float ty1 = fmul(fsub(ly, oy), iy), ty2 = fmul(fsub(hy, oy), iy);
    tmin = fmaxf(tmin, fminf(ty1, ty2));
    tmx = fminf(tmx, fmaxf(ty1, ty2));
    float tz1 = fmul(fsub(lz, oz), iz), tz2 = fmul(fsub(hz, oz), iz);
    tmin = fmaxf(tmin, fminf(tz1, tz2));
    tmx = fminf(tmx, fmaxf(tz1, tz2));
    float h = (tmin > 0) ? tmin : tmx;
    return tmx >= tmin && h >= 0 && h <= tmax;
}

// ----------------------------------------------------------- ErrorFloat sphere

struct EF {
    float v, e;
};
__device__ __forceinline__ EF ef_add(EF a, EF b) { return {fadd(a.v, b.v), fadd(a.e, b.e)}; }
__device__ __forceinline__ EF ef_sub(EF a, EF b) { return {fsub(a.v, b.v), fadd(a.e, b.e)}; }
__device__ __forceinline__ EF ef_mul(EF a, EF b)
{
    float v = fmul(a.v, b.v);
    return {v, fadd(fmul(fabsf(v), b.e), fmul(fabsf(b.v), a.e))};
}
__device__ __forceinline__ EF ef_smul(float s, EF b)
{
    float v = fmul(s, b.v);
    return {v, fmul(fabsf(v), b.e)};
}
__device__ __forceinline__ EF ef_div(EF a, EF b)
{
    float v = fdiv(a.v, b.v);
    return {v, fdiv(fadd(fmul(fabsf(v), b.e), fmul(fabsf(b.v), a.e)), fmul(b.v, b.v))};
}
__device__ __forceinline__ EF ef_sqrt(EF f)
{
    float v = __fsqrt_rn(f.v);
    return {v, __double2float_rn(__ddiv_rn(__dmul_rn(0.5, (double)f.e), (double)v))};
}

// Sphere::intersects (shapes/Sphere.cu:357-398) for a full sphere: ray to object space
// with error bounds (Transform.cu:328-404), normalized direction, ErrorFloat quadratic
// (math.cu:91-115), bound checks (Sphere.cu:41-81). Returns the object-space offset.
__device__ __forceinline__ bool sphere_test(const float *m, float radius, float ox, float oy, float oz, float dx,
                                            float dy, float dz, float tmax, float &tOut)
{
    const float eb3 = error_bound(3);
    float oe[3], de[3], po[3], pd[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const float *row = m + 4 * r;
        oe[r] = fmul(fadd(fadd(fadd(fabsf(fmul(row[0], ox)), fabsf(fmul(row[1], oy))), fabsf(fmul(row[2], oz))),
                          fabsf(row[3])),
                     eb3);
        de[r] = fmul(fadd(fadd(fabsf(fmul(row[0], dx)), fabsf(fmul(row[1], dy))), fabsf(fmul(row[2], dz))), eb3);
        po[r] = fadd(fadd(fadd(fmul(row[0], ox), fmul(row[1], oy)), fmul(row[2], oz)), row[3]);
        pd[r] = fadd(fadd(fmul(row[0], dx), fmul(row[1], dy)), fmul(row[2], dz));
    }
    float wp = fadd(fadd(fadd(fmul(m[12], ox), fmul(m[13], oy)), fmul(m[14], oz)), m[15]);
    float invw = fdiv(1.0f, wp);
#pragma unroll
    for (int r = 0; r < 3; r++) po[r] = fmul(invw, po[r]);
    float ls = fadd(fadd(fmul(pd[0], pd[0]), fmul(pd[1], pd[1])), fmul(pd[2], pd[2]));
    float tm = tmax;
    if (ls > 0) {
        float dt = fdiv(fadd(fadd(fmul(fabsf(pd[0]), oe[0]), fmul(fabsf(pd[1]), oe[1])), fmul(fabsf(pd[2]), oe[2])), ls);
#pragma unroll
        for (int r = 0; r < 3; r++) po[r] = fadd(po[r], fmul(pd[r], dt));
        tm = fsub(tm, dt);
    }
    float len = __fsqrt_rn(ls);
    float il = fdiv(1.0f, len);
#pragma unroll
    for (int r = 0; r < 3; r++) pd[r] = fmul(pd[r], il);
    EF eox = {po[0], oe[0]}, eoy = {po[1], oe[1]}, eoz = {po[2], oe[2]};
    EF edx = {pd[0], de[0]}, edy = {pd[1], de[1]}, edz = {pd[2], de[2]};
    EF a = ef_add(ef_add(ef_mul(edx, edx), ef_mul(edy, edy)), ef_mul(edz, edz));
    EF b = ef_smul(2.0f, ef_add(ef_add(ef_mul(edx, eox), ef_mul(edy, eoy)), ef_mul(edz, eoz)));
    EF c = ef_sub(ef_add(ef_add(ef_mul(eox, eox), ef_mul(eoy, eoy)), ef_mul(eoz, eoz)),
                  ef_mul(EF{radius, 0.f}, EF{radius, 0.f}));
    EF disc = ef_sub(ef_mul(b, b), ef_mul(ef_smul(4.0f, a), c));
    if (disc.v < 0.0f) return false;
    EF rd = ef_sqrt(disc);
    EF q = (b.v < 0.0f) ? ef_smul(-0.5f, ef_sub(b, rd)) : ef_smul(-0.5f, ef_add(b, rd));
    EF t0 = ef_div(q, a), t1 = ef_div(c, q);
    if (t0.v > t1.v) {
        EF tmp = t0;
        t0 = t1;
        t1 = tmp;
    }
    if (t0.v != t0.v || t0.e != t0.e || t1.v != t1.v || t1.e != t1.e) return false;
    if (fadd(t0.v, t0.e) > tm || fsub(t1.v, t1.e) <= 0) return false;
    EF th = t0;
    if (fsub(t0.v, t0.e) <= 0) {
        th = t1;
        if (fadd(t1.v, t1.e) > tm) return false;
    }
    tOut = th.v;
    return true;
}

// The world -> object transform of a ray as Transform::operator()(const Ray &) does it
// (Transform.cu:216-237): origin with its error bound, direction, origin moved to the edge of
// the bound (dt along the direction) and the limit reduced by dt. po / pd: object-space
// origin and direction, tm the reduced limit.
__device__ __forceinline__ void ray_to_object(const float *m, float ox, float oy, float oz, float dx, float dy, float dz,
                                              float tmax, float po[3], float pd[3], float &tm)
{
    const float eb3 = error_bound(3);
    float oe[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const float *row = m + 4 * r;
        oe[r] = fmul(fadd(fadd(fadd(fabsf(fmul(row[0], ox)), fabsf(fmul(row[1], oy))), fabsf(fmul(row[2], oz))),
                          fabsf(row[3])),
                     eb3);
        po[r] = fadd(fadd(fadd(fmul(row[0], ox), fmul(row[1], oy)), fmul(row[2], oz)), row[3]);
        pd[r] = fadd(fadd(fmul(row[0], dx), fmul(row[1], dy)), fmul(row[2], dz));
    }
    const float wp = fadd(fadd(fadd(fmul(m[12], ox), fmul(m[13], oy)), fmul(m[14], oz)), m[15]);
    const float invw = fdiv(1.0f, wp);
#pragma unroll
    for (int r = 0; r < 3; r++) po[r] = fmul(invw, po[r]);
    const float ls = fadd(fadd(fmul(pd[0], pd[0]), fmul(pd[1], pd[1])), fmul(pd[2], pd[2]));
    tm = tmax;
    if (ls > 0) {
        const float dt =
            fdiv(fadd(fadd(fmul(fabsf(pd[0]), oe[0]), fmul(fabsf(pd[1]), oe[1])), fmul(fabsf(pd[2]), oe[2])), ls);
#pragma unroll
        for (int r = 0; r < 3; r++) po[r] = fadd(po[r], fmul(pd[r], dt));
        tm = fsub(tm, dt);
    }
}

// Plane::intersects (shapes/Plane.cu:127-170): the ray in the plane's object space (its unit
// square [0,1]^2 at z = 0), skipped when |d.z| <= FLOAT_ERROR_MARGIN (1e-7, compared in double
// as the reference's double literal makes it); the hit point o - (o.z / d.z) d; the offset
// Ray::getOffset takes from the x components alone ((p.x - o.x) / d.x, so a ray whose
// object-space x direction is 0 never hits, Ray.cu:69-72); accepted when 0 < offset <= the
// world ray's limit and the point lies in the square. Returns the offset in tOut; uv: the
// object-space (x, y) (the surface point, Plane.cu:80-82).
__device__ __forceinline__ bool plane_test(const float *m, float ox, float oy, float oz, float dx, float dy, float dz,
                                           float tmax, float &tOut, float &u, float &v)
{
    float po[3], pd[3], tm;
    ray_to_object(m, ox, oy, oz, dx, dy, dz, tmax, po, pd, tm);
    if (!((double)fabsf(pd[2]) > 1e-7)) return false;
    const float s = fdiv(po[2], pd[2]);
    const float hx = fsub(po[0], fmul(s, pd[0])), hy = fsub(po[1], fmul(s, pd[1]));
    const float off = fmul(fsub(hx, po[0]), fdiv(1.0f, pd[0]));
    if (off <= 0.f || off > tmax || hx < 0.f || hx > 1.f || hy < 0.f || hy > 1.f) return false;
    if (!(off == off)) return false;  // NaN offsets fail the reference's offset < hitOffset test
    tOut = off;
    u = hx;
    v = hy;
    return true;
}

}  // namespace rtb
