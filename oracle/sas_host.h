/*
 * Host (C99) environment for sasmodels model sources in the oracle
 * restatement (test infrastructure only).
 *
 * Mirrors the C branch of the reference platform layer
 * (sasmodels/kernel_header.c:58-218): the same math-constant literals the
 * reference DLL sees under -std=c99 (kernel_header.c:144-169), the helper
 * functions the model C calls, and the storage words `constant`,
 * `pconstant`, `pglobal` reduced to plain C.
 */
#ifndef SAS_HOST_H
#define SAS_HOST_H

#include <stdint.h>
#include <math.h>

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

#define constant const
#define pconstant const
#define pglobal
#define SAS_DOUBLE double
#define powr(a, b) pow(a, b)
#define pown(a, b) pow(a, b)
#define SINCOS(angle, svar, cvar) \
    do { const double _a_ = (angle); svar = sin(_a_); cvar = cos(_a_); } while (0)

static inline double square(double x) { return x*x; }
static inline double cube(double x) { return x*x*x; }
static inline double clip(double x, double lo, double hi)
{
    return x < lo ? lo : (x > hi ? hi : x);
}
static inline double sas_sinx_x(double x) { return x == 0 ? 1.0 : sin(x)/x; }

static inline void SET_VEC(double *v, double a, double b, double c)
{
    v[0] = a; v[1] = b; v[2] = c;
}
static inline double SCALAR_VEC(const double *a, const double *b)
{
    return a[0]*b[0] + a[1]*b[1] + a[2]*b[2];
}
static inline void ORTH_VEC(double *r, const double *a, const double *b)
{
    const double s = SCALAR_VEC(a, b)/SCALAR_VEC(b, b);
    r[0] = a[0] - s*b[0];
    r[1] = a[1] - s*b[1];
    r[2] = a[2] - s*b[2];
}

#endif
