// Tone mapping of a film to 8-bit RGB: the reference's Film::toneMaxPixel operators
// (camera/Film.cu:156-282) restated on the GPU. The reference computes in double with a few
// float constants (its Float is float, types.h:22) promoted where its operators take Float;
// every such constant is written here as (double)(float)c, and every double operation is
// rounded on its own (no contraction), so the device result equals the reference's up to
// pow in gammaClamp.
#pragma once

#include <cstdint>

namespace rtb {

struct D3 {
    double r, g, b;
};

__host__ __device__ __forceinline__ double td_add(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ double td_sub(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ double td_mul(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double td_div(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

__host__ __device__ __forceinline__ D3 d3(double v) { return D3{v, v, v}; }
__host__ __device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{td_add(a.r, b.r), td_add(a.g, b.g), td_add(a.b, b.b)}; }
__host__ __device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{td_sub(a.r, b.r), td_sub(a.g, b.g), td_sub(a.b, b.b)}; }
__host__ __device__ __forceinline__ D3 operator*(D3 a, D3 b) { return D3{td_mul(a.r, b.r), td_mul(a.g, b.g), td_mul(a.b, b.b)}; }
__host__ __device__ __forceinline__ D3 operator/(D3 a, D3 b) { return D3{td_div(a.r, b.r), td_div(a.g, b.g), td_div(a.b, b.b)}; }
__host__ __device__ __forceinline__ D3 operator*(D3 a, double s) { return D3{td_mul(a.r, s), td_mul(a.g, s), td_mul(a.b, s)}; }
__host__ __device__ __forceinline__ D3 operator/(D3 a, double s) { return D3{td_div(a.r, s), td_div(a.g, s), td_div(a.b, s)}; }

// Spectrum::brightness (radiometry/Spectrum.cu:68-74): float weights held in doubles
__host__ __device__ __forceinline__ double tm_brightness(D3 p)
{
    const double wr = (double)0.212671f, wg = (double)0.715160f, wb = (double)0.072169f;
    return td_add(td_add(td_mul(wr, p.r), td_mul(wg, p.g)), td_mul(wb, p.b));
}

__host__ __device__ __forceinline__ double tm_clamp(double x, double a, double b) { return fmax(a, fmin(b, x)); }
__host__ __device__ __forceinline__ D3 tm_clamp(D3 p, double a, double b)
{
    return D3{tm_clamp(p.r, a, b), tm_clamp(p.g, a, b), tm_clamp(p.b, a, b)};
}

// uncharted2_tonemap_partial (Film.cu:194-203): A..F are floats; A*x promotes A, C*B and
// D*E, D*F, E/F are float products and quotients
__host__ __device__ __forceinline__ D3 tm_uncharted2_partial(D3 x)
{
    const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, F = 0.30f;
    const float cb = C * B, de = D * E, df = D * F, ef = E / F;
    return (x * ((x * (double)A) + d3((double)cb)) + d3((double)de)) / (x * ((x * (double)A) + d3((double)B)) + d3((double)df)) -
           d3((double)ef);
}

// rtt_and_odt_fit (Film.cu:216-221): 0.983729 * pixel goes through operator*(Float, Spectrum)
__host__ __device__ __forceinline__ D3 tm_rtt_odt(D3 p)
{
    const D3 a = p * (p + d3(0.0245786)) - d3(0.000090537);
    const D3 b = p * ((p * (double)0.983729f) + d3(0.4329510)) + d3(0.238081);
    return a / b;
}

__host__ __device__ __forceinline__ D3 tm_mat(const double m[9], D3 v)
{
    return D3{td_add(td_add(td_mul(m[0], v.r), td_mul(m[1], v.g)), td_mul(m[2], v.b)),
              td_add(td_add(td_mul(m[3], v.r), td_mul(m[4], v.g)), td_mul(m[5], v.b)),
              td_add(td_add(td_mul(m[6], v.r), td_mul(m[7], v.g)), td_mul(m[8], v.b))};
}

// Film::toneMaxPixel for a pixel sum over `samples` samples; maxc and maxl are the film's
// getMaxChannel and getMaxLuminance (already divided by the sample count).
__host__ __device__ inline D3 tonemap_pixel(D3 sum, double samples, double maxc, double maxl, uint32_t mode)
{
    D3 p = sum / samples;
    switch (mode) {
    case 0:  // equalize
        return p / maxc;
    case 1: {  // reinhard
        if (tm_brightness(p) == 0) return p;
        const double l_old = tm_brightness(p);
        const double numerator = td_mul(l_old, td_add(1.0, td_div(l_old, td_mul(maxl, maxl))));
        const double l_new = td_div(numerator, td_add(1.0, l_old));
        return tm_clamp(p * td_div(l_new, l_old), 0, 1);
    }
    case 2: {  // reinhardJodie: lerp(p / (1 + p), p / (1 + L), same) = (1 - x) * a + x * b
        const D3 rp = p / td_add(1.0, tm_brightness(p));
        const D3 x = p / (p + d3(1.0));
        return tm_clamp((d3(1.0) - x) * rp + x * rp, 0, 1);
    }
    case 3: {  // ACESfilmic
        const double in[9] = {0.59719, 0.35458, 0.04823, 0.07600, 0.90834, 0.01566, 0.02840, 0.13383, 0.83777};
        const double out[9] = {1.60475, -0.53108, -0.07367, -0.10208, 1.10813, -0.00605, -0.00327, -0.07276, 1.07602};
        return tm_clamp(tm_mat(out, tm_rtt_odt(tm_mat(in, p))), 0, 1);
    }
    case 4: {  // uncharted2 (exposure bias 2, white point 11.2; not clamped)
        const D3 curr = tm_uncharted2_partial(p * (double)2.0f);
        const D3 white_scale = d3(1.0) / tm_uncharted2_partial(d3(11.2));
        return curr * white_scale;
    }
    default: {  // gammaClamp: (p / max)^(1 / 2.2)
        const D3 q = p / maxc;
        const double e = td_div(1.0, 2.2);
        return D3{pow(q.r, e), pow(q.g, e), pow(q.b, e)};
    }
    }
}

// (unsigned char)(v * 255) as the reference's x86 build converts it: truncation to a 32-bit
// integer, then its low byte
__host__ __device__ __forceinline__ uint8_t tm_byte(double v) { return (uint8_t)(int32_t)td_mul(v, 255.0); }

}  // namespace rtb
