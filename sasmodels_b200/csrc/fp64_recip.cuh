// 1/d in FP64 by Newton's method, for the hoisted FP64 bindings: the
// hardware's approximate reciprocal (rcp.approx.ftz.f64) refined by two
// iterations x <- x + x (1 - d x), each squaring the relative error, to
// within an ulp or two of 1/d.  d must be a normal double (the seed flushes
// subnormals); every caller passes a value bounded away from zero.  Exact
// division when compiled for the host (the host checks of the bindings).
#pragma once

#ifdef __CUDACC__
__host__ __device__ __forceinline__
#else
inline
#endif
double recip_nr(double d)
{
#ifdef __CUDA_ARCH__
    double x;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(d));
    double e = fma(-d, x, 1.0);
    x = fma(x, e, x);
    e = fma(-d, x, 1.0);
    return fma(x, e, x);
#else
    return 1.0/d;
#endif
}
