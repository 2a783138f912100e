// Device-side environment for sasmodels model C sources.
//
// Model plugins (sasmodels/models/*.c and models/lib/*.c) are written against
// a small platform layer (sasmodels/kernel_header.c).  This header provides
// that layer for sm_100a device code so the model sources compile unchanged
// as __device__ functions:
//   - the helpers they call: square, cube, clip, sas_sinx_x, SINCOS, powr/pown
//     and the SET_VEC/SCALAR_VEC/ORTH_VEC vector helpers used by the
//     magnetic driver (kernel_header.c:170-218);
//   - the storage-class words they use: `constant` (tables and pointers to
//     them; the generator rewrites file-scope tables as __device__ const),
//     `pconstant`, `pglobal`;
//   - the math constants the reference DLL sees.  The DLL is compiled with
//     -std=c99, where glibc's math.h does not define M_PI and friends, so
//     the DLL uses the literals of kernel_header.c:144-169.  Some are not the
//     correctly rounded value (M_PI_2, M_SQRT1_2, M_4PI_3); they are
//     reproduced here digit for digit so the GPU evaluates the same formula.
#pragma once

#include <cstdint>
#include <cmath>

#include "fp64_recip.cuh"

#undef M_PI
#undef M_PI_2
#undef M_PI_4
#undef M_E
#undef M_SQRT1_2
#define M_PI 3.141592653589793
#define M_PI_2 1.570796326794897
#define M_PI_4 0.7853981633974483
#define M_E 2.718281828459045091
#define M_SQRT1_2 0.70710678118654746
#define M_PI_180 0.017453292519943295
#define M_4PI_3 4.18879020478639

#define pglobal
#define pconstant const
#define SAS_DOUBLE double

#define SINCOS(angle, svar, cvar) sincos((angle), &(svar), &(cvar))
#define powr(a, b) pow(a, b)
#define pown(a, b) pow(a, b)

__device__ __forceinline__ double square(double x) { return x*x; }
__device__ __forceinline__ double cube(double x) { return x*x*x; }
__device__ __forceinline__ float square(float x) { return x*x; }
__device__ __forceinline__ float cube(float x) { return x*x*x; }
// numpy.clip semantics: NaN propagates (kernel_header.c:172-176)
__device__ __forceinline__ double clip(double x, double low, double high)
{
    return x < low ? low : (x > high ? high : x);
}
__device__ __forceinline__ double sas_sinx_x(double x)
{
    return x == 0 ? 1.0 : sin(x)/x;
}

__device__ __forceinline__ void SET_VEC(double *v, double a, double b, double c)
{
    v[0] = a; v[1] = b; v[2] = c;
}
__device__ __forceinline__ double SCALAR_VEC(const double *a, const double *b)
{
    return a[0]*b[0] + a[1]*b[1] + a[2]*b[2];
}
__device__ __forceinline__ void ORTH_VEC(double *r, const double *a, const double *b)
{
    const double s = SCALAR_VEC(a, b)/SCALAR_VEC(b, b);
    r[0] = a[0] - s*b[0];
    r[1] = a[1] - s*b[1];
    r[2] = a[2] - s*b[2];
}
