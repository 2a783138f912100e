// Resolution smearing on the GPU, the step that follows the kernel in every
// fit (sasmodels/direct_model.py:345 -> Resolution.apply).
//
//   pinhole_smear       1D pinhole (sasmodels/resolution.py:172-220): each
//                       measured q_i averages the theory over the calculated
//                       points q_calc[j] within [q_i - 2.5 s_i, q_i + 3 s_i],
//                       weighted by the gaussian mass of each point's bin,
//                       erf((e[j+1] - q_i)/(sqrt2 s_i)) - erf((e[j] - q_i)/(sqrt2 s_i)),
//                       normalised by the weights' sum.  The reference builds
//                       the dense n_calc x nq matrix and multiplies; here one
//                       warp per q_i walks only its band (computed on the host
//                       by binary search), forming the weights on the fly: the
//                       work is the band, not the matrix.
//   slit_smear          1D slit (sasmodels/resolution.py:223-395): per q_i
//                       and per step across the slit width, the bins between
//                       |q| and sqrt(q^2 + l^2) found by binary search, the
//                       u-substituted bin widths formed on the fly.
//   nllf_sets           the fit objective of every curve of a population
//                       against one data set (bumps_model.py:263-282).
//   pinhole2d_average   2D pinhole (sasmodels/resolution2d.py:162-175): the
//                       weighted average over the nbins oversampling points of
//                       every q, products and sums rounded separately in bin
//                       order, as numpy's axis-0 reduction does.
//
// Both read theory values the model kernel left on the device, so a fit step
// needs no host round trip between the kernel and the smearing.
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace res {

constexpr unsigned FULL = 0xffffffffu;
constexpr double SQRT2 = 1.4142135623730951;     // numpy sqrt(2.0), correctly rounded

// One curve per blockIdx.y: theory + y*theory_stride -> out + y*out_stride.
__global__ void __launch_bounds__(256)
pinhole_smear(int nq, const double *__restrict__ q, const double *__restrict__ width,
              const int32_t *__restrict__ lo, const int32_t *__restrict__ hi,
              const double *__restrict__ edges, const double *__restrict__ theory,
              double *__restrict__ out, size_t theory_stride, size_t out_stride)
{
    const int i = (int)((blockIdx.x*(size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= nq) return;                      // whole warps leave together
    theory += blockIdx.y*theory_stride;
    out += blockIdx.y*out_stride;
    const double qi = q[i];
    const double s = SQRT2*width[i];
    double acc = 0.0, wsum = 0.0;
    for (int j = lo[i] + lane; j < hi[i]; j += 32) {
        const double w = erf((edges[j + 1] - qi)/s) - erf((edges[j] - qi)/s);
        acc += w*theory[j];
        wsum += w;
    }
    #pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc += __shfl_xor_sync(FULL, acc, off);
        wsum += __shfl_xor_sync(FULL, wsum, off);
    }
    if (lane == 0) out[i] = acc/wsum;
}

__global__ void __launch_bounds__(256)
pinhole2d_average(int nq, int nbins, const double *__restrict__ theory,
                  const double *__restrict__ weights, double wsum, double *__restrict__ out)
{
    const int i = (int)(blockIdx.x*(size_t)blockDim.x + threadIdx.x);
    if (i >= nq) return;
    double num = __dmul_rn(theory[i], weights[0]);
    for (int b = 1; b < nbins; ++b)
        num = __dadd_rn(num, __dmul_rn(theory[(size_t)b*nq + i], weights[b]));
    out[i] = num/wsum;
}

// Binary search: first index in edges[0..n) with edges[k] >= x (or > x
// when strict), the same in every lane.
__device__ __forceinline__ int lower_edge(const double *edges, int n, double x, bool strict)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const bool before = strict ? edges[mid] <= x : edges[mid] < x;
        if (before) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// u(e) of the slit integral (sasmodels/resolution.py:387-395): e^2 - q^2
// inside [|q|, sqrt(q^2 + l^2)], 0 below, (limit^2 - q^2) above.  Each
// product and difference is rounded on its own (no contraction into an
// FMA): sqrt(u) near the lower limit amplifies the last bit of u.
__device__ __forceinline__ double sq_diff(double a, double b)
{
    return __dsub_rn(__dmul_rn(a, a), __dmul_rn(b, b));
}

__device__ __forceinline__ double slit_u(double e, double qk, double limit)
{
    if (e < fabs(qk)) return 0.0;
    if (e > limit) return sq_diff(limit, qk);
    return sq_diff(e, qk);
}

__global__ void __launch_bounds__(256)
slit_smear(int nq, int n_calc, const double *__restrict__ q, const double *__restrict__ width,
           const double *__restrict__ length, int n_length, const double *__restrict__ q_calc,
           const double *__restrict__ edges, const double *__restrict__ theory,
           double *__restrict__ out)
{
    const int i = (int)((blockIdx.x*(size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= nq) return;
    const double qi = q[i], wi = width[i], li = length[i];
    double acc = 0.0;
    if (wi == 0.0 && li == 0.0) {
        // perfect resolution: the theory at q_calc == q
        for (int j = lane; j < n_calc; j += 32)
            if (q_calc[j] == qi) acc += theory[j];
    } else {
        const int kmax = wi == 0.0 ? 0 : n_length;
        for (int k = -kmax; k <= kmax; ++k) {
            const double qk = kmax ? qi + (k*wi)/n_length : qi;
            const double limit = sqrt(__dadd_rn(__dmul_rn(qk, qk), __dmul_rn(li, li)));
            // bins whose u changes: from the last edge below |qk| to the
            // first edge above the limit
            const int a = max(lower_edge(edges, n_calc + 1, fabs(qk), false) - 1, 0);
            const int b = min(lower_edge(edges, n_calc + 1, limit, true), n_calc);
            for (int j = a + lane; j < b; j += 32) {
                const double w = __dsub_rn(sqrt(slit_u(edges[j + 1], qk, limit)),
                                           sqrt(slit_u(edges[j], qk, limit)))/li;
                acc += w*theory[j];
            }
        }
        acc /= (double)(2*kmax + 1);
    }
    #pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(FULL, acc, off);
    if (lane == 0) out[i] = acc;
}

// Negative log-likelihood of each curve against one data set
// (bumps_model.py:263-282): 0.5 sum_i ((theory_i - y_i)/dy_i)^2, one block
// per curve, a fixed-order tree over its points.
__global__ void __launch_bounds__(256)
nllf_sets(int nq, const double *__restrict__ theory, size_t theory_stride,
          const double *__restrict__ y, const double *__restrict__ dy, double *__restrict__ out)
{
    const double *th = theory + blockIdx.x*theory_stride;
    double acc = 0.0;
    for (int i = threadIdx.x; i < nq; i += 256) {
        const double r = (th[i] - y[i])/dy[i];
        acc += r*r;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    for (int s = 128; s > 0; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    }
    if (threadIdx.x == 0) out[blockIdx.x] = 0.5*red[0];
}

inline char *errbuf()
{
    static thread_local char buf[256] = "";
    return buf;
}

inline int32_t status(const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::snprintf(errbuf(), 256, "%s: %s", what, cudaGetErrorString(e));
        return -3;
    }
    return 0;
}

}  // namespace res

extern "C" {

const char *sasb200_resolution_last_error(void) { return res::errbuf(); }

// out[nq] = smeared theory; lo/hi: band [lo_i, hi_i) of calculated points of
// each q (0 <= lo_i <= hi_i <= n_calc); edges[n_calc + 1]; theory[n_calc].
int32_t sasb200_pinhole_smear(int32_t nq, int32_t n_calc, const double *q, const double *width,
                              const int32_t *lo, const int32_t *hi, const double *edges,
                              const double *theory, double *out, void *stream)
{
    res::errbuf()[0] = 0;
    if (nq < 0 || n_calc < 0 || (nq > 0 && (!q || !width || !lo || !hi || !edges || !theory
                                            || !out)))
        return (std::snprintf(res::errbuf(), 256, "bad arguments"), -1);
    if (nq == 0) return 0;
    const int threads = 256;
    const long long warps = nq;
    const unsigned blocks = (unsigned)((warps*32 + threads - 1)/threads);
    res::pinhole_smear<<<blocks, threads, 0, (cudaStream_t)stream>>>(nq, q, width, lo, hi,
                                                                      edges, theory, out, 0, 0);
    return res::status("pinhole_smear");
}

// The same smearing for n_sets curves at once (a fit population sharing one
// data set): theory[s*theory_stride + j], out[s*out_stride + i].
int32_t sasb200_pinhole_smear_sets(int32_t n_sets, int32_t nq, int32_t n_calc, const double *q,
                                   const double *width, const int32_t *lo, const int32_t *hi,
                                   const double *edges, const double *theory,
                                   int64_t theory_stride, double *out, int64_t out_stride,
                                   void *stream)
{
    res::errbuf()[0] = 0;
    if (n_sets < 0 || n_sets > 65535 || nq < 0 || n_calc < 0 || theory_stride < n_calc
        || out_stride < nq || (nq > 0 && n_sets > 0 && (!q || !width || !lo || !hi || !edges
                                                          || !theory || !out)))
        return (std::snprintf(res::errbuf(), 256, "bad arguments"), -1);
    if (nq == 0 || n_sets == 0) return 0;
    const int threads = 256;
    const dim3 grid((unsigned)(((long long)nq*32 + threads - 1)/threads), (unsigned)n_sets);
    res::pinhole_smear<<<grid, threads, 0, (cudaStream_t)stream>>>(
        nq, q, width, lo, hi, edges, theory, out, (size_t)theory_stride, (size_t)out_stride);
    return res::status("pinhole_smear_sets");
}

// out[s] = 0.5 sum_i ((theory[s*theory_stride + i] - y[i])/dy[i])^2.
int32_t sasb200_nllf_sets(int32_t n_sets, int32_t nq, const double *theory,
                          int64_t theory_stride, const double *y, const double *dy,
                          double *out, void *stream)
{
    res::errbuf()[0] = 0;
    if (n_sets < 0 || nq < 0 || theory_stride < nq
        || (n_sets > 0 && (!theory || !y || !dy || !out)))
        return (std::snprintf(res::errbuf(), 256, "bad arguments"), -1);
    if (n_sets == 0) return 0;
    res::nllf_sets<<<n_sets, 256, 0, (cudaStream_t)stream>>>(nq, theory, (size_t)theory_stride,
                                                              y, dy, out);
    return res::status("nllf_sets");
}

// Slit smearing: out[i] = sum_j W[i, j] theory[j] with the slit weights of
// sasmodels/resolution.py:223-395 (length only, or width and length with
// 2 n_length + 1 steps across the width); q_calc[n_calc] sorted, edges
// [n_calc + 1].  A nonzero width with a zero length is refused on the host,
// as by the reference.
int32_t sasb200_slit_smear(int32_t nq, int32_t n_calc, const double *q, const double *width,
                           const double *length, int32_t n_length, const double *q_calc,
                           const double *edges, const double *theory, double *out,
                           void *stream)
{
    res::errbuf()[0] = 0;
    if (nq < 0 || n_calc < 0 || n_length < 1 || (nq > 0 && (!q || !width || !length || !q_calc
                                                             || !edges || !theory || !out)))
        return (std::snprintf(res::errbuf(), 256, "bad arguments"), -1);
    if (nq == 0) return 0;
    const int threads = 256;
    const unsigned blocks = (unsigned)(((long long)nq*32 + threads - 1)/threads);
    res::slit_smear<<<blocks, threads, 0, (cudaStream_t)stream>>>(
        nq, n_calc, q, width, length, n_length, q_calc, edges, theory, out);
    return res::status("slit_smear");
}

// out[nq] = sum_b weights[b] theory[b*nq + i] / wsum, bins in order.
int32_t sasb200_pinhole2d_average(int32_t nq, int32_t nbins, const double *theory,
                                  const double *weights, double wsum, double *out, void *stream)
{
    res::errbuf()[0] = 0;
    if (nq < 0 || nbins < 1 || (nq > 0 && (!theory || !weights || !out)))
        return (std::snprintf(res::errbuf(), 256, "bad arguments"), -1);
    if (nq == 0) return 0;
    const int threads = 256;
    res::pinhole2d_average<<<(nq + threads - 1)/threads, threads, 0, (cudaStream_t)stream>>>(
        nq, nbins, theory, weights, wsum, out);
    return res::status("pinhole2d_average");
}

}  // extern "C"
