// Throughput probes for the roofline denominators of the sasmodels kernels.
//
// The hot path is bound by the FP64 pipe (FP64 form) or by FP32 FMA plus the
// transcendental unit (FP32 forms), not by HBM or tensor cores, so the
// roofline needs those peaks measured on the same part at the same clocks.
// Each probe runs independent dependency chains per thread (enough to cover
// pipe latency) and writes one value per thread so nothing is dead code.
//
//   sasb200_probe_fp64_fma(out, blocks, iters, stream): 16 chains of DFMA
//       2 flops per DFMA; flops = blocks*256*16*iters*2
//   sasb200_probe_fp32_fma(out, blocks, iters, stream): 16 chains of FFMA
//   sasb200_probe_mufu_sin(out, blocks, iters, stream): 16 chains of
//       __sinf (MUFU.SIN); ops = blocks*256*16*iters
//
// All pointers are device pointers; out needs blocks*256 elements.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

constexpr int THREADS = 256;
constexpr int CHAINS = 16;

__global__ void __launch_bounds__(THREADS) fp64_fma(double *out, int iters, double b, double c)
{
    double a[CHAINS];
    #pragma unroll
    for (int k = 0; k < CHAINS; ++k) a[k] = threadIdx.x*1e-3 + k;
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int k = 0; k < CHAINS; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
    #pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += a[k];
    out[blockIdx.x*THREADS + threadIdx.x] = s;
}

__global__ void __launch_bounds__(THREADS) fp32_fma(float *out, int iters, float b, float c)
{
    float a[CHAINS];
    #pragma unroll
    for (int k = 0; k < CHAINS; ++k) a[k] = threadIdx.x*1e-3f + k;
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int k = 0; k < CHAINS; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.0f;
    #pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += a[k];
    out[blockIdx.x*THREADS + threadIdx.x] = s;
}

__global__ void __launch_bounds__(THREADS) mufu_sin(float *out, int iters)
{
    float a[CHAINS];
    #pragma unroll
    for (int k = 0; k < CHAINS; ++k) a[k] = threadIdx.x*1e-3f + k*0.1f;
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int k = 0; k < CHAINS; ++k) a[k] = __sinf(a[k]);
    }
    float s = 0.0f;
    #pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += a[k];
    out[blockIdx.x*THREADS + threadIdx.x] = s;
}

}  // namespace

extern "C" int32_t sasb200_probe_fp64_fma(double *out, int32_t blocks, int32_t iters, void *stream)
{
    fp64_fma<<<blocks, THREADS, 0, (cudaStream_t)stream>>>(out, iters, 0.999999, 1e-7);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

extern "C" int32_t sasb200_probe_fp32_fma(float *out, int32_t blocks, int32_t iters, void *stream)
{
    fp32_fma<<<blocks, THREADS, 0, (cudaStream_t)stream>>>(out, iters, 0.999f, 1e-4f);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

extern "C" int32_t sasb200_probe_mufu_sin(float *out, int32_t blocks, int32_t iters, void *stream)
{
    mufu_sin<<<blocks, THREADS, 0, (cudaStream_t)stream>>>(out, iters);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

extern "C" int32_t sasb200_probe_threads_per_block(void) { return THREADS; }
extern "C" int32_t sasb200_probe_chains(void) { return CHAINS; }
