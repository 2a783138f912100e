// Special functions for the FP32-compensated form.
//
// Bulk arithmetic runs in FP32 and on the transcendental unit (MUFU);
// only the phase of each oscillating factor is formed and reduced in FP64.
// An FP32 argument q*r of a few hundred carries an absolute phase error of
// ~1e-5 rad, which on its own would put the orientation/size averages
// ~1e-4 away from the FP64 result; an FP64 phase reduced modulo 2*pi and then
// handed to FP32 keeps them within a few 1e-7.
//
// Functions (x is the FP64 argument, results are FP32):
//   sph_j1c_f(x)   3 j1(x)/x            (sas_3j1x_x.c:46-57)
//   j1c_f(x)       2 J1(x)/x            (sas_J1.c:155-245, single precision)
//   sinc_f(x)      sin(x)/x             (kernel_header.c:177)
//
// Series branches cover the small-argument region where the closed forms
// cancel; their cut-offs are set so each branch is accurate to ~1e-7
// relative in FP32.
#pragma once

#include <cstdint>

namespace f32c {

// 2*pi split into a double head and the residual of the double rounding
constexpr double TWO_PI_HI = 6.283185307179586;
constexpr double TWO_PI_LO = 2.4492935982947064e-16;
constexpr double INV_TWO_PI = 0.15915494309189535;
constexpr double THREE_PI_4 = 2.356194490192345;

// x - 2*pi*k with k = nearest integer to x/(2*pi); |result| <= pi (plus a
// few ulp).  Cody-Waite with a two-part constant: exact enough in FP64 for
// |x| up to ~1e6, far beyond q*size in SAS.
__device__ __forceinline__ float reduce_2pi(double x)
{
    const double k = rint(x*INV_TWO_PI);
    const double r = fma(-k, TWO_PI_HI, x) - k*TWO_PI_LO;
    return (float)r;
}

// 1/x on the MUFU unit, without the round-to-nearest correction (relative
// error about one FP32 ulp, far inside the form's 1e-5); x is a normal
// float here (|x| >= 1 at every call).
__device__ __forceinline__ float rcp_f(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sin and cos of a reduced phase |r| <= ~pi + 0.3 on the MUFU unit.
// Absolute error <= 2^-21.4 on [-pi, pi].
__device__ __forceinline__ void sincos_reduced(float r, float &s, float &c)
{
    __sincosf(r, &s, &c);
}

// 3 j1(x)/x.  Taylor series 3 sum_k (-1)^k x^2k / ((2k+3)!! (2k)!!) for
// |x| < 1.5 (7 terms, truncation < 5e-9); closed form 3(sin x/x - cos x)/x^2
// beyond, where the cancellation costs at most a factor ~3.
__device__ __forceinline__ float sph_j1c_f(double x)
{
    const float xf = (float)x;
    const float ax = fabsf(xf);
    if (ax < 1.5f) {
        const float t = xf*xf;
        return 1.0f + t*(-1.0f/10.0f + t*(1.0f/280.0f + t*(-1.0f/15120.0f
               + t*(1.0f/1330560.0f + t*(-1.0f/172972800.0f
               + t*(1.0f/31135104000.0f))))));
    }
    float s, c;
    sincos_reduced(reduce_2pi(x), s, c);
    const float inv = rcp_f(xf);
    return 3.0f*(s*inv - c)*inv*inv;
}

// sin(x)/x.  Series 1 - x^2/6 + ... to x^10 for |x| < 1 (truncation
// < 2e-10), reduced-phase MUFU sine beyond.
__device__ __forceinline__ float sinc_f(double x)
{
    const float xf = (float)x;
    if (fabsf(xf) < 1.0f) {
        const float t = xf*xf;
        return 1.0f + t*(-1.0f/6.0f + t*(1.0f/120.0f + t*(-1.0f/5040.0f
               + t*(1.0f/362880.0f + t*(-1.0f/39916800.0f)))));
    }
    float s, c;
    sincos_reduced(reduce_2pi(x), s, c);
    return s*rcp_f(xf);
}

// Single-precision Bessel J1 after Cephes j1f (S. L. Moshier, Cephes Math
// Library 2.2, j1f.c), as used by sasmodels' FP32 kernels (sas_J1.c:155-231):
// for |x| <= 2 a polynomial in x^2 times x (x^2 - z1); beyond, the
// asymptotic amplitude sqrt(1/x) P(1/x) and phase x - 3pi/4 + (1/x) Q(1/x^2).
// Here the x - 3pi/4 part of the phase is taken in FP64 and reduced, the
// small correction added in FP32.  Returns 2 J1(x)/x (1 at x = 0).
__device__ __forceinline__ float j1c_f(double x)
{
    // published Cephes j1f coefficients (highest power first)
    const float z1 = 1.46819706421238932572e1f;
    const double ax = fabs(x);
    const float axf = (float)ax;
    if (axf <= 2.0f) {
        const float z = axf*axf;
        float p = -4.878788132172128e-09f;
        p = p*z + 6.009061827883699e-07f;
        p = p*z - 4.541343896997497e-05f;
        p = p*z + 1.937383947804541e-03f;
        p = p*z - 3.405537384615824e-02f;
        // J1(x) = (z - z1) x p ; 2 J1(x)/x = 2 (z - z1) p
        return axf == 0.0f ? 1.0f : 2.0f*(z - z1)*p;
    }
    const float q = rcp_f(axf);
    float m = 6.913942741265801e-02f;
    m = m*q - 2.284801500053359e-01f;
    m = m*q + 3.138238455499697e-01f;
    m = m*q - 2.102302420403875e-01f;
    m = m*q + 5.435364690523026e-03f;
    m = m*q + 1.493389585089498e-01f;
    m = m*q + 4.976029650847191e-06f;
    m = m*q + 7.978845453073848e-01f;
    const float w = q*q;
    float ph = -4.497014141919556e+01f;
    ph = ph*w + 5.073465654089319e+01f;
    ph = ph*w - 2.485774108720340e+01f;
    ph = ph*w + 7.222973196770240e+00f;
    ph = ph*w - 1.544842782180211e+00f;
    ph = ph*w + 3.503787691653334e-01f;
    ph = ph*w - 1.637986776941202e-01f;
    ph = ph*w + 3.749989509080821e-01f;
    const float phase = reduce_2pi(ax - THREE_PI_4) + q*ph;
    float s, c;
    sincos_reduced(phase, s, c);
    const float amp = sqrtf(q)*m;
    return 2.0f*amp*c*q;            // 2 J1(x)/x, even in x
}

// FP64 square root from an FP32 reciprocal-square-root seed and one
// Newton-Raphson correction (relative error ~1e-14, enough for a phase).
__device__ __forceinline__ double sqrt_d_fast(double a)
{
    if (!(a > 0.0)) return 0.0;
    const double y = (double)rsqrtf((float)a);
    const double s0 = a*y;
    return fma(0.5*y, fma(-s0, s0, a), s0);
}

}  // namespace f32c
