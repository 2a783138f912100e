// Batched 1D evaluation of a whole fit population in one persistent launch.
//
// A bumps/DREAM population is thousands of parameter sets of one model, each
// with its own q vector and dispersity mesh.  The reference evaluates them
// one DLL call at a time (bumps_model.py:250-261 -> direct_model.py:319-351
// -> Kernel.Fq); here all sets are packed into flat arrays and cut on the
// host into work items
//
//     item = (set, 32-q tile, mesh range [m0, m1))
//
// of roughly equal cost, sorted longest first.  A persistent grid of warps
// pulls items from an atomic counter.  Inside an item the warp walks the mesh
// points; for each point and each of its 32 q:
//   * short quadratures (<= SHORT_RULE points) run one q per lane;
//   * long ones (500 / 5000 points) are spread over the 32 lanes of the
//     warp, one q at a time, and reduced with a shuffle butterfly,
// so lanes neither diverge on the rule length nor sit idle on small sets.
// Per-item FP64 partial sums are combined per (set, tile) in mesh order by
// batch_finalize, which also applies the normalisation of Kernel.Iq
// (kernel.py:80-99) to give I(q) per set.  Every sum has a fixed order.
//
// Flat layouts (all device memory):
//   sets   int32[8*n_sets]  nq, q_off, det_off, val_off, num_eval, raw_off,
//                           iq_off, tile_off
//   items  int32[4*n_items] set, q0, m0, m1
//   tile_items_off int32[n_tiles+1], tile_items int32[n_items]: items of each
//          (set, tile) in mesh order; tile index = sets[tile_off] + q0/32
//   partials float64[64*n_items]: F^2 then F sums of the item's 32 q
//   norms  float64[4*n_sets], raw float64[sum(2 nq + 4)], iq float64[sum nq]
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sasb200 {

constexpr int SHORT_RULE = 76;
constexpr int SET_FIELDS = 8;
constexpr int ITEM_FIELDS = 4;

// Whole plugin Fq as a single "node": the FP64 form evaluates each q in one
// lane with the model's own quadrature loop.
template <class M>
struct QuadWhole {
    struct S { double q; double v[M::NPARS > 0 ? M::NPARS : 1]; };
    __device__ static S setup(double q, const double *v)
    {
        S s;
        s.q = q;
        #pragma unroll
        for (int k = 0; k < M::NPARS; ++k) s.v[k] = v[k];
        return s;
    }
    __device__ static int nodes(const S &) { return 1; }
    __device__ static void node(const S &s, int, double &t1, double &t2)
    {
        double F1, F2;
        M::fq(s.q, F1, F2, s.v);
        t1 += F1;
        t2 += F2;
    }
    __device__ static void finish(const S &, double t1, double t2, double &F1, double &F2)
    {
        F1 = t1;
        F2 = t2;
    }
};

// One oriented 2D evaluation per (q, mesh point) along the qx axis (qy = 0)
// at the set's own view angles: the line cut of a 2D pattern without
// orientation dispersion, for models with an Iqac kernel.  The rotation and
// the qab/qc split are those of the Iqxy kernel (mesh_prepare + eval_2d,
// kernel_iq.c:197-242) with zero jitter, so a set gives what the 2D kernel
// gives for q vectors (q, 0).
template <class M>
struct QuadLine {
    struct S { double qab, qc; double v[M::NPARS > 0 ? M::NPARS : 1]; };
    __device__ static S setup(double q, const double *v, const double *values)
    {
        S s;
        #pragma unroll
        for (int k = 0; k < M::NPARS; ++k) s.v[k] = v[k];
        double rot[2];
        rotation_ac(values[M::THETA_PAR + 2], values[M::THETA_PAR + 3],
                    v[M::THETA_PAR], v[M::THETA_PAR + 1], rot);
        const double qx = q, qy = 0.0;
        s.qc = rot[0]*qx + rot[1]*qy;
        const double qab_sq = -s.qc*s.qc + qx*qx + qy*qy;
        s.qab = qab_sq > 0.0 ? sqrt(qab_sq) : 0.0;
        return s;
    }
    __device__ static int nodes(const S &) { return 1; }
    __device__ static void node(const S &s, int, double &, double &t2)
    {
        t2 += M::iqac(s.qab, s.qc, s.v);
    }
    __device__ static void finish(const S &, double, double t2, double &F1, double &F2)
    {
        F1 = 0.0;
        F2 = t2;
    }
};

// Q::setup(q, v, values) where the functor takes the set's values (QuadLine),
// Q::setup(q, v) otherwise.
template <class Q>
__device__ __forceinline__ auto quad_setup(double q, const double *v, const double *values, int)
    -> decltype(Q::setup(q, v, values))
{
    return Q::setup(q, v, values);
}

template <class Q>
__device__ __forceinline__ typename Q::S quad_setup(double q, const double *v, const double *,
                                                    long)
{
    return Q::setup(q, v);
}

// Parameters and weight of 1D mesh point `step` (same rule as mesh_prepare
// for the Iq kernel: outermost-first weight product, VALID, cutoff).
template <class M>
__device__ __forceinline__ bool mesh_point_1d(const int32_t *det, const double *values,
                                              int step, double cutoff, double *v, double &w)
{
    constexpr int MPD = M::MAX_PD;
    const DetailsView<MPD> d{det};
    #pragma unroll
    for (int k = 0; k < M::NPARS; ++k) v[k] = values[2 + k];
    const double *pd_value = values + M::NVALUES;
    const double *pd_weight = pd_value + d.num_weights();
    double weight = 1.0;
    #pragma unroll
    for (int k = MPD - 1; k >= 0; --k) {
        const int n = max(d.pd_length(k), 1);
        const int i = (step/max(d.pd_stride(k), 1)) % n;
        const int off = d.pd_offset(k) + i;
        const int p = d.pd_par(k);
        const double pv = pd_value[off];
        #pragma unroll
        for (int j = 0; j < M::NPARS; ++j) if (j == p) v[j] = pv;
        weight = pd_weight[off]*weight;
    }
    w = weight;
    return M::valid(v) && weight > cutoff;
}

template <class M>
__global__ void __launch_bounds__(128)
batch_norms(int n_sets, const int32_t *__restrict__ sets, const int32_t *__restrict__ det_all,
            const double *__restrict__ val_all, double cutoff, int reff_mode,
            double *__restrict__ norms)
{
    const int set = blockIdx.x;
    if (set >= n_sets) return;
    const int32_t *sd = sets + SET_FIELDS*set;
    const int32_t *det = det_all + sd[2];
    const double *values = val_all + sd[3];
    const int num_eval = sd[4];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    double v[M::NPARS > 0 ? M::NPARS : 1];
    for (int m = threadIdx.x; m < num_eval; m += 128) {
        double w;
        if (!mesh_point_1d<M>(det, values, m, cutoff, v, w)) continue;
        double form, shell;
        M::volume(v, form, shell);
        a[0] += w;
        a[1] += w*form;
        a[2] += w*shell;
        if (reff_mode != 0) a[3] += w*M::reff(reff_mode, v);
    }
    __shared__ double red[4][128];
    #pragma unroll
    for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = a[k];
    for (int s = 64; s > 0; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) {
            #pragma unroll
            for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        }
    }
    if (threadIdx.x == 0) {
        #pragma unroll
        for (int k = 0; k < 4; ++k) norms[4*set + k] = red[k][0];
    }
}

template <class M, class Q, int WARPS>
__global__ void __launch_bounds__(32*WARPS)
batch_main(int n_items, const int32_t *__restrict__ items, const int32_t *__restrict__ sets,
           const double *__restrict__ q_all, const int32_t *__restrict__ det_all,
           const double *__restrict__ val_all, double cutoff,
           double *__restrict__ partials, int *__restrict__ counter)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(counter, 1);
        item = __shfl_sync(FULL_MASK, item, 0);
        if (item >= n_items) break;
        const int32_t *it = items + ITEM_FIELDS*item;
        const int32_t *sd = sets + SET_FIELDS*it[0];
        const int q0 = it[1], m0 = it[2], m1 = it[3];
        const int nq = sd[0];
        const double *q = q_all + sd[1];
        const int32_t *det = det_all + sd[2];
        const double *values = val_all + sd[3];
        const bool q_ok = q0 + lane < nq;
        const double qk = q[q_ok ? q0 + lane : q0];
        double acc2 = 0.0, acc1 = 0.0;
        double v[M::NPARS > 0 ? M::NPARS : 1];
        for (int m = m0; m < m1; ++m) {
            double w;
            if (!mesh_point_1d<M>(det, values, m, cutoff, v, w)) continue;   // warp-uniform
            typename Q::S s = quad_setup<Q>(qk, v, values, 0);
            const int n = q_ok ? Q::nodes(s) : 0;
            const bool shortq = n <= SHORT_RULE;
            if (q_ok && shortq) {
                double t1 = 0.0, t2 = 0.0;
                for (int i = 0; i < n; ++i) Q::node(s, i, t1, t2);
                double F1, F2;
                Q::finish(s, t1, t2, F1, F2);
                acc2 += w*F2;
                acc1 += w*F1;
            }
            unsigned longq = __ballot_sync(FULL_MASK, q_ok && !shortq);
            while (longq) {
                const int L = __ffs(longq) - 1;
                longq &= longq - 1;
                const double qL = __shfl_sync(FULL_MASK, qk, L);
                const typename Q::S sL = quad_setup<Q>(qL, v, values, 0);
                const int nL = Q::nodes(sL);
                double t1 = 0.0, t2 = 0.0;
                for (int i = lane; i < nL; i += 32) Q::node(sL, i, t1, t2);
                #pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    t1 += __shfl_xor_sync(FULL_MASK, t1, off);
                    t2 += __shfl_xor_sync(FULL_MASK, t2, off);
                }
                if (lane == L) {
                    double F1, F2;
                    Q::finish(sL, t1, t2, F1, F2);
                    acc2 += w*F2;
                    acc1 += w*F1;
                }
            }
        }
        partials[64*(size_t)item + lane] = acc2;
        partials[64*(size_t)item + 32 + lane] = acc1;
    }
}

template <class M>
__global__ void __launch_bounds__(128)
batch_finalize(int n_sets, const int32_t *__restrict__ sets,
               const int32_t *__restrict__ tile_items_off, const int32_t *__restrict__ tile_items,
               const double *__restrict__ partials, const double *__restrict__ norms,
               const double *__restrict__ val_all, double *__restrict__ raw_all,
               double *__restrict__ iq_all)
{
    const int set = blockIdx.x;
    if (set >= n_sets) return;
    const int32_t *sd = sets + SET_FIELDS*set;
    const int nq = sd[0];
    const double *values = val_all + sd[3];
    double *raw = raw_all + sd[5];
    double *iq = iq_all + sd[6];
    const double *nm = norms + 4*set;
    // Kernel.Fq normalisation (kernel.py:172-188)
    double total = nm[0];
    if (total == 0.0) total = 1.0;
    double shell = nm[2]/total;
    if (shell == 0.0) shell = 1.0;
    const double scale = values[0], background = values[1];
    for (int qi = threadIdx.x; qi < nq; qi += 128) {
        const int tile = sd[7] + qi/32;
        double F2 = 0.0, F1 = 0.0;
        for (int k = tile_items_off[tile]; k < tile_items_off[tile + 1]; ++k) {
            const double *p = partials + 64*(size_t)tile_items[k];
            F2 += p[qi % 32];
            F1 += p[32 + qi % 32];
        }
        raw[2*qi] = F2;
        raw[2*qi + 1] = F1;
        iq[qi] = (scale/shell)*(F2/total) + background;
    }
    if (threadIdx.x < 4) raw[2*nq + threadIdx.x] = nm[threadIdx.x];
}

template <class M, class Q, int WARPS>
__host__ int32_t batch_launch(int32_t n_sets, const int32_t *sets, const double *q_all,
                              const int32_t *det_all, const double *val_all, int32_t n_items,
                              const int32_t *items, const int32_t *tile_items_off,
                              const int32_t *tile_items, double cutoff, int32_t reff_mode,
                              double *partials, double *norms, double *raw_all,
                              double *iq_all, int32_t *counter, int32_t blocks,
                              cudaStream_t st)
{
    if (blocks <= 0) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_main<M, Q, WARPS>,
                                                      32*WARPS, 0);
        blocks = device_sms()*(per_sm > 0 ? per_sm : 1);
    }
    cudaMemsetAsync(counter, 0, sizeof(int32_t), st);
    batch_norms<M><<<n_sets, 128, 0, st>>>(n_sets, sets, det_all, val_all, cutoff,
                                           reff_mode, norms);
    if (n_items > 0) {
        batch_main<M, Q, WARPS><<<blocks, 32*WARPS, 0, st>>>(
            n_items, items, sets, q_all, det_all, val_all, cutoff, partials, counter);
    }
    batch_finalize<M><<<n_sets, 128, 0, st>>>(n_sets, sets, tile_items_off, tile_items,
                                              partials, norms, val_all, raw_all, iq_all);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        std::snprintf(error_buffer(), 256, "batch launch: %s", cudaGetErrorString(err));
        return ERR_CUDA;
    }
    return OK;
}

template <class M, class Q>
__host__ int32_t batch_dispatch(int32_t warps, int32_t n_sets, const int32_t *sets,
                                const double *q_all, const int32_t *det_all,
                                const double *val_all, int32_t n_items, const int32_t *items,
                                const int32_t *tile_items_off, const int32_t *tile_items,
                                double cutoff, int32_t reff_mode, double *partials,
                                double *norms, double *raw_all, double *iq_all,
                                int32_t *counter, int32_t blocks, cudaStream_t st)
{
    switch (warps) {
    case 4:
        return batch_launch<M, Q, 4>(n_sets, sets, q_all, det_all, val_all, n_items, items,
                                     tile_items_off, tile_items, cutoff, reff_mode, partials,
                                     norms, raw_all, iq_all, counter, blocks, st);
    case 8:
        return batch_launch<M, Q, 8>(n_sets, sets, q_all, det_all, val_all, n_items, items,
                                     tile_items_off, tile_items, cutoff, reff_mode, partials,
                                     norms, raw_all, iq_all, counter, blocks, st);
    default:
        return fail(ERR_ARGUMENT, "warps per block must be 4 or 8");
    }
}

// Line form (QuadLine) where the model has an Iqac kernel.
template <class M>
__host__ int32_t batch_dispatch_line(int32_t warps, int32_t n_sets, const int32_t *sets,
                                     const double *q_all, const int32_t *det_all,
                                     const double *val_all, int32_t n_items,
                                     const int32_t *items, const int32_t *tile_items_off,
                                     const int32_t *tile_items, double cutoff,
                                     int32_t reff_mode, double *partials, double *norms,
                                     double *raw_all, double *iq_all, int32_t *counter,
                                     int32_t blocks, cudaStream_t st)
{
    if constexpr (M::XY_MODE == XY_QAC) {
        return batch_dispatch<M, QuadLine<M>>(warps, n_sets, sets, q_all, det_all, val_all,
                                              n_items, items, tile_items_off, tile_items,
                                              cutoff, reff_mode, partials, norms, raw_all,
                                              iq_all, counter, blocks, st);
    } else {
        return fail(ERR_ARGUMENT, "the line form needs a model with an Iqac kernel");
    }
}

}  // namespace sasb200

// int32 sasb200_<name>_batch(form, warps, blocks, n_sets, sets, q_all, det_all,
//     val_all, n_items, items, tile_items_off, tile_items, cutoff,
//     reff_mode, partials, norms, raw_all, iq_all, counter, stream)
// form 0 = FP64 (the plugin's own Fq per lane), 1 = FP32-compensated;
// 2 / 3 = the line form (QuadLine: 2D along qx at the set's view angles,
// no orientation dispersion) in FP64 / FP32-compensated.
#define SASB200_EXPORT_BATCH(NAME, MODEL64, MODEL32)                                     \
extern "C" int32_t sasb200_##NAME##_batch(                                              \
    int32_t form, int32_t warps, int32_t blocks, int32_t n_sets, const int32_t *sets,   \
    const double *q_all, const int32_t *det_all, const double *val_all,                 \
    int32_t n_items, const int32_t *items, const int32_t *tile_items_off,               \
    const int32_t *tile_items, double cutoff, int32_t reff_mode, double *partials,      \
    double *norms, double *raw_all, double *iq_all, int32_t *counter, void *stream)     \
{                                                                                       \
    sasb200::error_buffer()[0] = 0;                                                     \
    if (n_sets < 0 || n_items < 0 || !sets || !counter)                                 \
        return sasb200::fail(sasb200::ERR_ARGUMENT, "bad batch arguments");             \
    if (n_sets == 0) return 0;                                                          \
    cudaStream_t st = static_cast<cudaStream_t>(stream);                                \
    if (form == 0)                                                                      \
        return sasb200::batch_dispatch<MODEL64, sasb200::QuadWhole<MODEL64>>(           \
            warps, n_sets, sets, q_all, det_all, val_all, n_items, items,               \
            tile_items_off, tile_items, cutoff, reff_mode, partials, norms, raw_all,    \
            iq_all, counter, blocks, st);                                               \
    if (form == 1)                                                                      \
        return sasb200::batch_dispatch<MODEL32, MODEL32::Quad>(                \
            warps, n_sets, sets, q_all, det_all, val_all, n_items, items,               \
            tile_items_off, tile_items, cutoff, reff_mode, partials, norms, raw_all,    \
            iq_all, counter, blocks, st);                                               \
    if (form == 2 || form == 3)                                                         \
        return form == 2                                                                \
            ? sasb200::batch_dispatch_line<MODEL64>(                                    \
                  warps, n_sets, sets, q_all, det_all, val_all, n_items, items,         \
                  tile_items_off, tile_items, cutoff, reff_mode, partials, norms,       \
                  raw_all, iq_all, counter, blocks, st)                                 \
            : sasb200::batch_dispatch_line<MODEL32>(                                    \
                  warps, n_sets, sets, q_all, det_all, val_all, n_items, items,         \
                  tile_items_off, tile_items, cutoff, reff_mode, partials, norms,       \
                  raw_all, iq_all, counter, blocks, st);                                \
    return sasb200::fail(sasb200::ERR_ARGUMENT, "form must be 0..3");                   \
}
