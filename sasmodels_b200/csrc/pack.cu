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
//   * dispersed (sasmodels/weights.py:21-220, 264-291): sigma = width*value
//     for a volume parameter (centre = value) or width for an orientation
//     jitter (centre 0); the points are numpy.linspace(start, stop, N) with
//         gaussian, rectangle, lognormal, schulz, boltzmann:
//             x_i = centre + linspace(-nsigma*sigma, nsigma*sigma, N)_i
//         uniform:
//             x_i = linspace(centre - sigma, centre + sigma, N)_i
//     linspace_i = i*step + start, step = (stop - start)/(N - 1), the last
//     point = stop; of these the points inside the parameter's limits (and,
//     for the rectangle, within |sigma| sqrt(3) of the centre) are kept: a
//     contiguous index range [first, first + npts) that the host computes
//     with the same arithmetic.  Densities (unnormalised):
//         gaussian   exp((x - c)^2 / ((-2 sigma) sigma))
//         uniform, rectangle   1
//         lognormal  exp(-0.5 ((log x - log c)/s)^2)/(x s), s = |sigma/c|
//         schulz     exp(z log z + (z - 1) log(x/c) - (x/c) z - log c - lgamma z),
//                    z = (c/sigma)^2
//         boltzmann  exp(-|x - c|/|sigma|)
//     normalised by their sum in numpy's pairwise order.  Every product,
//     quotient and sum is rounded on its own as numpy rounds it, so the
//     points are bit for bit the host's; exp, log and lgamma may differ from
//     numpy's and scipy's by an ulp or two.
// Magnetic sets (magnetic[s] != 0) then have their (M0, mtheta, mphi)
// triples turned into (mx, my, mz) = M0 (sin t cos p, sin t sin p, cos t)
// in place, as details.py:288-306 does.
// Sets the table cannot describe are marshaled on the host and skipped here
// (val_off < 0).
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace pk {

constexpr int MAX_PARS = 64;      // kernel parameters of one model
constexpr int COMMON = 2;         // scale, background precede the kernel parameters
constexpr int FLAG_RELATIVE = 1;  // width is relative to the value
constexpr int FLAG_KEEP = 2;      // an idle parameter keeps its value (else 0)

// distribution codes of the kinds table
enum Kind { GAUSSIAN = 0, UNIFORM = 1, RECTANGLE = 2, LOGNORMAL = 3, SCHULZ = 4,
            BOLTZMANN = 5 };
constexpr double DEG = 0.017453292519943295;   // numpy.radians factor pi/180

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

// Unnormalised density of distribution `kind` at x (see the file comment).
__device__ __forceinline__ double density(int kind, double x, double c, double sigma)
{
    switch (kind) {
    case GAUSSIAN: {
        const double d = __dsub_rn(x, c);
        return exp(__ddiv_rn(__dmul_rn(d, d), __dmul_rn(__dmul_rn(-2.0, sigma), sigma)));
    }
    case LOGNORMAL: {
        const double s = fabs(__ddiv_rn(sigma, c));
        const double t = __ddiv_rn(__dsub_rn(log(x), log(c)), s);
        return __ddiv_rn(exp(__dmul_rn(-0.5, __dmul_rn(t, t))), __dmul_rn(x, s));
    }
    case SCHULZ: {
        const double R = __ddiv_rn(x, c);
        const double q = __ddiv_rn(c, sigma);
        const double z = __dmul_rn(q, q);
        double a = __dmul_rn(z, log(z));
        a = __dadd_rn(a, __dmul_rn(__dsub_rn(z, 1.0), log(R)));
        a = __dsub_rn(a, __dmul_rn(R, z));
        a = __dsub_rn(a, log(c));
        a = __dsub_rn(a, lgamma(z));
        return exp(a);
    }
    case BOLTZMANN:
        return exp(__ddiv_rn(-fabs(__dsub_rn(x, c)), fabs(sigma)));
    default:            // uniform, rectangle
        return 1.0;
    }
}

// One block per set.
__global__ void __launch_bounds__(128)
pack_values(int n_sets, int nvalues, int npars, int nmag,
            const double *__restrict__ scalars, const double *__restrict__ widths,
            const double *__restrict__ nsigmas, const int32_t *__restrict__ npts,
            const int32_t *__restrict__ first, const int32_t *__restrict__ ntot,
            const int32_t *__restrict__ kinds, const int32_t *__restrict__ flags,
            const int32_t *__restrict__ magnetic, const int64_t *__restrict__ val_off,
            const int64_t *__restrict__ val_size, double *__restrict__ values)
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
    const int32_t *fst = first + (size_t)s*npars;
    const int32_t *tot = ntot + (size_t)s*npars;
    const int32_t *knd = kinds + (size_t)s*npars;
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
    if (magnetic[s] && threadIdx.x == 0) {
        // (M0, mtheta, mphi) -> (mx, my, mz) in place (details.py:288-306)
        for (int m = 0; m < nmag; ++m) {
            double *t = v + nvalues - 3*nmag + 3*m;
            const double M0 = t[0];
            const double th = __dmul_rn(t[1], DEG), ph = __dmul_rn(t[2], DEG);
            const double Ms = __dmul_rn(M0, sin(th));
            t[0] = __dmul_rn(Ms, cos(ph));
            t[1] = __dmul_rn(Ms, sin(ph));
            t[2] = __dmul_rn(M0, cos(th));
        }
    }
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
        const int kind = knd[k];
        const bool relative = f & FLAG_RELATIVE;
        const double sigma = relative ? __dmul_rn(wid[k], value) : wid[k];
        const double center = relative ? value : 0.0;
        // numpy.linspace(lo, hi, N), added to the centre except for uniform
        const bool flat = kind == UNIFORM;
        const double lo = flat ? __dsub_rn(center, sigma) : __dmul_rn(-nsg[k], sigma);
        const double hi = flat ? __dadd_rn(center, sigma) : __dmul_rn(nsg[k], sigma);
        const int N = tot[k];
        const double delta = __dsub_rn(hi, lo);
        const double div = (double)(N - 1);
        const double step = __ddiv_rn(delta, div);
        double *x = xs + start[k];
        double *w = ws + start[k];
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int i = fst[k] + j;
            double y = step == 0.0 ? __dmul_rn(__ddiv_rn((double)i, div), delta)
                                   : __dmul_rn((double)i, step);
            y = __dadd_rn(y, lo);
            if (i == N - 1) y = hi;
            const double xi = flat ? y : __dadd_rn(center, y);
            x[j] = xi;
            w[j] = density(kind, xi, center, sigma);
        }
        __syncthreads();
        if (threadIdx.x == 0) total = pairwise_sum(w, n);
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) w[j] = __ddiv_rn(w[j], total);
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

int32_t sasb200_pack_values(int32_t n_sets, int32_t nvalues, int32_t npars, int32_t nmag,
                            const double *scalars, const double *widths, const double *nsigmas,
                            const int32_t *npts, const int32_t *first, const int32_t *ntot,
                            const int32_t *kinds, const int32_t *flags,
                            const int32_t *magnetic, const int64_t *val_off,
                            const int64_t *val_size, double *values, void *stream)
{
    pk::errbuf()[0] = 0;
    if (n_sets < 0 || npars < 0 || npars > pk::MAX_PARS || nmag < 0
        || nvalues < pk::COMMON + npars + 3*nmag)
        return (std::snprintf(pk::errbuf(), 256, "bad sizes"), -1);
    if (n_sets == 0) return 0;
    if (!scalars || !val_off || !val_size || !values || !magnetic
        || (npars > 0 && (!widths || !nsigmas || !npts || !first || !ntot || !kinds
                          || !flags)))
        return (std::snprintf(pk::errbuf(), 256, "null pointer"), -1);
    pk::pack_values<<<(unsigned)n_sets, 128, 0, (cudaStream_t)stream>>>(
        n_sets, nvalues, npars, nmag, scalars, widths, nsigmas, npts, first, ntot, kinds,
        flags, magnetic, val_off, val_size, values);
    return pk::status("pack_values");
}

}  // extern "C"
