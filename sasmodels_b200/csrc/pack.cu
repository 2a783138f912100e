// Device-side marshaling of a fit population: the values vector of every
// parameter set (sasmodels/details.py:225-254, make_kernel_args) built on the
// GPU from a compact per-set table, so that a new generation of a fit crosses
// PCIe as a few numbers per set instead of its dispersity meshes.
//
// Values layout of one set (padded with zeros to a multiple of 32):
//
//     [ scalars (nvalues) | x_0 .. x_{npars-1} | w_0 .. w_{npars-1} | 0 ... ]
//
// where (x_k, w_k) is the dispersity mesh of kernel parameter k:
//   * idle (no dispersity): one point, the parameter's value (or 0 for an
//     orientation jitter), weight 1;
//   * gaussian (sasmodels/weights.py:78-83, 86-102, 264-291):
//         sigma = width*center (volume parameters) or width (orientation
//         jitter, centred on 0),
//         x_i = center + (i*step + start), start = -nsigma*sigma,
//         stop = nsigma*sigma, step = (stop - start)/(n - 1), x_{n-1} = center + stop
//         (numpy.linspace),
//         w_i = exp((x_i - center)^2/((-2 sigma) sigma))/sum_j(...),
//     every product, quotient and sum rounded on its own as numpy rounds it,
//     the sum in numpy's pairwise order.  Only exp may differ from the host
//     (by an ulp or two).
// Sets whose points would be clipped at a parameter limit, or whose mesh is
// not gaussian, are marshaled on the host and skipped here (val_off < 0).
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace pk {

constexpr int MAX_PARS = 64;      // kernel parameters of one model
constexpr int COMMON = 2;         // scale, background precede the kernel parameters
constexpr int FLAG_RELATIVE = 1;  // width is relative to the value
constexpr int FLAG_KEEP = 2;      // an idle parameter keeps its value (else 0)

// numpy's pairwise summation of a contiguous float64 row (add.reduce):
// fewer than 8 terms summed in order from -0.0; up to 128 terms in eight
// interleaved partial sums combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)),
// then the remainder in order; longer rows split at n/2 rounded down to a
// multiple of 8 and the halves added.  Iterative over an explicit stack.
__device__ double pairwise_sum(const double *a, int n)
{
    struct Part { int start, n, state; double left; };
    Part stack[32];                    // depth log2(n/128) + 1 < 32
    int top = 0;
    stack[0] = {0, n, 0, 0.0};
    double ret = 0.0;
    while (top >= 0) {
        Part &p = stack[top];
        if (p.n <= 128) {
            const double *x = a + p.start;
            double res;
            if (p.n < 8) {
                res = -0.0;
                for (int i = 0; i < p.n; ++i) res = __dadd_rn(res, x[i]);
            } else {
                double r[8];
                for (int j = 0; j < 8; ++j) r[j] = x[j];
                int i = 8;
                for (; i < p.n - (p.n % 8); i += 8)
                    for (int j = 0; j < 8; ++j) r[j] = __dadd_rn(r[j], x[i + j]);
                res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                                __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
                for (; i < p.n; ++i) res = __dadd_rn(res, x[i]);
            }
            ret = res;
            --top;
        } else if (p.state == 0) {           // descend into the left half
            int n2 = p.n/2;
            n2 -= n2 % 8;
            p.state = 1;
            stack[top + 1] = {p.start, n2, 0, 0.0};
            ++top;
            continue;
        } else if (p.state == 1) {           // left done: descend into the right half
            int n2 = p.n/2;
            n2 -= n2 % 8;
            p.left = ret;
            p.state = 2;
            stack[top + 1] = {p.start + n2, p.n - n2, 0, 0.0};
            ++top;
            continue;
        } else {
            ret = __dadd_rn(p.left, ret);
            --top;
        }
        // a finished part hands `ret` to its parent, which resumes at its state
    }
    return ret;
}

// One block per set.
__global__ void __launch_bounds__(128)
pack_values(int n_sets, int nvalues, int npars, const double *__restrict__ scalars,
            const double *__restrict__ widths, const double *__restrict__ nsigmas,
            const int32_t *__restrict__ npts, const int32_t *__restrict__ flags,
            const int64_t *__restrict__ val_off, const int64_t *__restrict__ val_size,
            double *__restrict__ values)
{
    const int s = blockIdx.x;
    if (s >= n_sets) return;
    const int64_t off = val_off[s];
    if (off < 0) return;                      // marshaled on the host
    double *v = values + off;
    const double *row = scalars + (size_t)s*nvalues;
    const double *wid = widths + (size_t)s*npars;
    const double *nsg = nsigmas + (size_t)s*npars;
    const int32_t *np_ = npts + (size_t)s*npars;
    __shared__ int start[MAX_PARS + 1];
    __shared__ double total;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < npars; ++k) {
            start[k] = acc;
            acc += np_[k] > 0 ? np_[k] : 1;
        }
        start[npars] = acc;
    }
    for (int j = threadIdx.x; j < nvalues; j += blockDim.x) v[j] = row[j];
    __syncthreads();
    const int len = start[npars];
    double *xs = v + nvalues;
    double *ws = v + nvalues + len;
    for (int k = 0; k < npars; ++k) {
        const int n = np_[k];
        const double value = row[COMMON + k];
        const int f = flags[k];
        if (n <= 0) {
            if (threadIdx.x == 0) {
                xs[start[k]] = (f & FLAG_KEEP) ? value : 0.0;
                ws[start[k]] = 1.0;
            }
            continue;
        }
        const bool relative = f & FLAG_RELATIVE;
        const double sigma = relative ? __dmul_rn(wid[k], value) : wid[k];
        const double center = relative ? value : 0.0;
        const double lo = __dmul_rn(-nsg[k], sigma);
        const double hi = __dmul_rn(nsg[k], sigma);
        const double delta = __dsub_rn(hi, lo);
        const double div = (double)(n - 1);
        const double step = __ddiv_rn(delta, div);
        const double den = __dmul_rn(__dmul_rn(-2.0, sigma), sigma);
        double *x = xs + start[k];
        double *w = ws + start[k];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double y = step == 0.0 ? __dmul_rn(__ddiv_rn((double)i, div), delta)
                                   : __dmul_rn((double)i, step);
            y = __dadd_rn(y, lo);
            if (i == n - 1) y = hi;
            const double xi = __dadd_rn(center, y);
            const double d = __dsub_rn(xi, center);
            x[i] = xi;
            w[i] = exp(__ddiv_rn(__dmul_rn(d, d), den));
        }
        __syncthreads();
        if (threadIdx.x == 0) total = pairwise_sum(w, n);
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] = __ddiv_rn(w[i], total);
        __syncthreads();
    }
    const int64_t used = nvalues + 2*(int64_t)len;
    for (int64_t j = used + threadIdx.x; j < val_size[s]; j += blockDim.x) v[j] = 0.0;
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

}  // namespace pk

extern "C" {

const char *sasb200_pack_last_error(void) { return pk::errbuf(); }

int32_t sasb200_pack_max_pars(void) { return pk::MAX_PARS; }

int32_t sasb200_pack_values(int32_t n_sets, int32_t nvalues, int32_t npars,
                            const double *scalars, const double *widths, const double *nsigmas,
                            const int32_t *npts, const int32_t *flags, const int64_t *val_off,
                            const int64_t *val_size, double *values, void *stream)
{
    pk::errbuf()[0] = 0;
    if (n_sets < 0 || npars < 0 || npars > pk::MAX_PARS || nvalues < pk::COMMON + npars)
        return (std::snprintf(pk::errbuf(), 256, "bad sizes"), -1);
    if (n_sets == 0) return 0;
    if (!scalars || !val_off || !val_size || !values
        || (npars > 0 && (!widths || !nsigmas || !npts || !flags)))
        return (std::snprintf(pk::errbuf(), 256, "null pointer"), -1);
    pk::pack_values<<<(unsigned)n_sets, 128, 0, (cudaStream_t)stream>>>(
        n_sets, nvalues, npars, scalars, widths, nsigmas, npts, flags, val_off, val_size, values);
    return pk::status("pack_values");
}

}  // extern "C"
