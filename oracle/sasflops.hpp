/*
 * SAS-flop counting arithmetic (measurement infrastructure only: it sizes
 * the roofline numerator; nothing on the product path uses it).
 *
 * The reference's model C is compiled as C++ with `double` replaced by the
 * value type `SF` below.  Every SF operation computes the IEEE double result
 * it would have computed and adds its cost under the "SAS-flop v1"
 * convention to a per-thread counter, so running the reference's own model
 * code on the configuration's own inputs replays every branch it takes
 * (J1 small/large argument, the 3j1(x)/x series cutoff, the adaptive Gauss
 * rule length, x == 0 guards) and counts exactly the operations of the
 * branches taken.
 *
 * SAS-flop v1 (a counting convention, not a model of any library):
 *   +, -, *                          1
 *   compare (<, >, <=, >=, ==, !=)   1
 *   fabs, fmin, fmax                 1   (compare/select)
 *   /                                4
 *   sqrt                             4
 *   sin, cos, exp, log, cbrt, asin,
 *   acos, atan                       16
 *   sincos (the SINCOS macro)        24
 *   pow                              32  (exp + log)
 *   unary minus                      0   (a sign flip)
 * A source `a*b + c` therefore counts 2.
 *
 * The math-constant literals are the reference platform's
 * (sasmodels/kernel_header.c:144-169), as in sas_host.h.
 */
#ifndef SASFLOPS_HPP
#define SASFLOPS_HPP

#include <cmath>
#include <cstdint>
#include <cstring>

namespace sasflops {
extern thread_local uint64_t count;
}

#define SF_INLINE static inline __attribute__((always_inline))

struct SF {
    double v;
    SF() = default;
    constexpr SF(double x) : v(x) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
};

SF_INLINE SF operator+(SF a, SF b) { ++sasflops::count; return SF(a.v + b.v); }
SF_INLINE SF operator-(SF a, SF b) { ++sasflops::count; return SF(a.v - b.v); }
SF_INLINE SF operator*(SF a, SF b) { ++sasflops::count; return SF(a.v * b.v); }
SF_INLINE SF operator/(SF a, SF b) { sasflops::count += 4; return SF(a.v / b.v); }
SF_INLINE SF operator-(SF a) { return SF(-a.v); }
SF_INLINE SF operator+(SF a) { return a; }
SF_INLINE SF &operator+=(SF &a, SF b) { a = a + b; return a; }
SF_INLINE SF &operator-=(SF &a, SF b) { a = a - b; return a; }
SF_INLINE SF &operator*=(SF &a, SF b) { a = a * b; return a; }
SF_INLINE SF &operator/=(SF &a, SF b) { a = a / b; return a; }
SF_INLINE bool operator<(SF a, SF b) { ++sasflops::count; return a.v < b.v; }
SF_INLINE bool operator>(SF a, SF b) { ++sasflops::count; return a.v > b.v; }
SF_INLINE bool operator<=(SF a, SF b) { ++sasflops::count; return a.v <= b.v; }
SF_INLINE bool operator>=(SF a, SF b) { ++sasflops::count; return a.v >= b.v; }
SF_INLINE bool operator==(SF a, SF b) { ++sasflops::count; return a.v == b.v; }
SF_INLINE bool operator!=(SF a, SF b) { ++sasflops::count; return a.v != b.v; }

SF_INLINE SF sin(SF x) { sasflops::count += 16; return SF(std::sin(x.v)); }
SF_INLINE SF cos(SF x) { sasflops::count += 16; return SF(std::cos(x.v)); }
SF_INLINE SF exp(SF x) { sasflops::count += 16; return SF(std::exp(x.v)); }
SF_INLINE SF log(SF x) { sasflops::count += 16; return SF(std::log(x.v)); }
SF_INLINE SF cbrt(SF x) { sasflops::count += 16; return SF(std::cbrt(x.v)); }
SF_INLINE SF asin(SF x) { sasflops::count += 16; return SF(std::asin(x.v)); }
SF_INLINE SF acos(SF x) { sasflops::count += 16; return SF(std::acos(x.v)); }
SF_INLINE SF atan(SF x) { sasflops::count += 16; return SF(std::atan(x.v)); }
SF_INLINE SF sqrt(SF x) { sasflops::count += 4; return SF(std::sqrt(x.v)); }
SF_INLINE SF pow(SF x, SF y) { sasflops::count += 32; return SF(std::pow(x.v, y.v)); }
SF_INLINE SF fabs(SF x) { ++sasflops::count; return SF(std::fabs(x.v)); }
SF_INLINE SF fmax(SF a, SF b) { ++sasflops::count; return SF(std::fmax(a.v, b.v)); }
SF_INLINE SF fmin(SF a, SF b) { ++sasflops::count; return SF(std::fmin(a.v, b.v)); }

#define SINCOS(angle, svar, cvar) \
    do { const SF _a_ = (angle); sasflops::count += 24; \
         svar = SF(std::sin(_a_.v)); cvar = SF(std::cos(_a_.v)); } while (0)

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
#define powr(a, b) pow(a, b)
#define pown(a, b) pow(a, b)

/* From here on the model sources see SF wherever they say double. */
#define double SF
#define SAS_DOUBLE SF

static inline double square(double x) { return x*x; }
static inline double cube(double x) { return x*x*x; }
static inline double clip(double x, double lo, double hi)
{
    return x < lo ? lo : (x > hi ? hi : x);
}
static inline double sas_sinx_x(double x) { return x == 0 ? SF(1.0) : sin(x)/x; }

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
