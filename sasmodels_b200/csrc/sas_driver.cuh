// B200 polydispersity / orientation / magnetism driver.
//
// Replaces the generic kernel driver of the reference (sasmodels/kernel_iq.c)
// for one model M (a SasModel binding struct emitted by the generator).  The
// computation is the same weighted sum,
//
//     result[q]      = sum_{mesh points k, weight_k > cutoff, VALID}  w_k F^2(q; p_k)
//     result[tail+0] = sum_k w_k,   tail+1: sum_k w_k V_form,
//     tail+2: sum_k w_k V_shell,    tail+3: sum_k w_k R_eff
//
// but organised for the GPU in three launches instead of one thread per q
// walking the whole mesh:
//
//   1. mesh_prepare  one thread per mesh point decodes the mixed-radix index,
//                    forms the weight product, applies VALID, the jitter
//                    projection and the cutoff, accumulates the volume norms,
//                    builds the per-point rotation, and writes the surviving
//                    points compacted into 128-point segments of an
//                    array-of-structs table [weight, p[0..NPARS), rotation].
//   2. iq_main       q tiles map to thread blocks.  Within a warp LQ lanes take
//                    LQ neighbouring q and the 32/LQ lane groups take different
//                    mesh points; the WARPS warps of a block interleave over
//                    the segment, which is staged in shared memory.  FP64
//                    partial sums are reduced with warp shuffles, then across
//                    warps through shared memory, then written per mesh split.
//   3. finalize      sums the mesh splits in a fixed order and the segment
//                    norms in a fixed tree, and writes (or, for a restarted
//                    call, adds to) the result vector.
//
// Every reduction has a fixed order that depends only on the tile shape, so a
// call is bitwise reproducible.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sasb200 {

enum Variant { VAR_IQ = 0, VAR_IQXY = 1, VAR_IMAGNETIC = 2 };
enum XYMode { XY_1D = 0, XY_QA = 1, XY_QAC = 2, XY_QABC = 3, XY_QXY = 4 };

// Mesh points per segment (and threads per mesh_prepare block).
constexpr int SEG = 128;
constexpr unsigned FULL_MASK = 0xffffffffu;

// Mixed-radix mesh descriptor, the int32 CallDetails buffer
// (kernel_iq.c:47-58, details.py:43-113) for a model with MPD pd slots.
template <int MPD>
struct DetailsView {
    const int32_t *buf;
    __device__ int pd_par(int d) const { return buf[d]; }
    __device__ int pd_length(int d) const { return buf[MPD + d]; }
    __device__ int pd_offset(int d) const { return buf[2*MPD + d]; }
    __device__ int pd_stride(int d) const { return buf[3*MPD + d]; }
    __device__ int num_eval() const { return buf[4*MPD]; }
    __device__ int num_weights() const { return buf[4*MPD + 1]; }
    __device__ int theta_par() const { return buf[4*MPD + 3]; }
};

// A binding may restate one 2D form of its model with the per-mesh-point
// invariants hoisted out of the q loop: it declares `HOIST` (the XY mode it
// covers), `NH` (doubles per table row), `hoist_row(weight, v, rot, row)`
// (run once per kept mesh point by mesh_prepare) and
// `eval_row(qx, qy, qsq, row)` (returns weight * F^2 for one q).  Bindings
// without these keep the generic [weight, v, rotation] rows.
template <class M, class = void>
struct hoist_mode { static constexpr int value = 0; };
template <class M>
struct hoist_mode<M, decltype((void)M::HOIST, void())> {
    static constexpr int value = M::HOIST;
};
template <class M, class = void>
struct hoist_width { static constexpr int value = 1; };
template <class M>
struct hoist_width<M, decltype((void)M::NH, void())> {
    static constexpr int value = M::NH;
};

// A binding may also evaluate all spin channels of the magnetic variant at
// once (`MAG_FUSED`, `mag_channels(q, v, eff, chan_w)` for models without
// orientation), sharing the channel-independent factors of its amplitude.
template <class M, class = void>
struct mag_fused { static constexpr bool value = false; };
template <class M>
struct mag_fused<M, decltype((void)M::MAG_FUSED, void())> {
    static constexpr bool value = M::MAG_FUSED;
};
template <class M, bool ON>
struct MagOps {
    template <class E>
    __device__ static double channels(double, const double *, const E &, const double *)
    {
        return 0.0;
    }
};
template <class M>
struct MagOps<M, true> {
    template <class E>
    __device__ static double channels(double q, const double *v, const E &eff,
                                      const double *chan_w)
    {
        return M::mag_channels(q, v, eff, chan_w);
    }
};

// Per-variant table layout.
template <class M, int VAR>
struct Layout {
    static constexpr int XY = (VAR == VAR_IQ) ? XY_1D : M::XY_MODE;
    static constexpr int NROT = (XY == XY_QAC) ? 2 : (XY == XY_QABC) ? 6 : 0;
    static constexpr int NP = M::NPARS > 0 ? M::NPARS : 1;
    static constexpr bool HOISTED = (VAR == VAR_IQXY) && hoist_mode<M>::value == XY
                                    && XY != XY_1D;
    static constexpr int NF = HOISTED ? ((hoist_width<M>::value + 1) & ~1)
                                      : ((1 + M::NPARS + NROT) + 1) & ~1;  // 16-byte rows
    static constexpr bool FQ1D = (VAR == VAR_IQ) && M::HAVE_FQ;
    static constexpr int NOUT = FQ1D ? 2 : 1;
};

// Hoisted-row hooks, reached only when Layout<M, VAR>::HOISTED.
template <class M, bool ON>
struct HoistOps {
    __device__ static void row(double, const double *, const double *, double *) {}
    __device__ static double eval(double, double, double, const double *) { return 0.0; }
};
template <class M>
struct HoistOps<M, true> {
    __device__ static void row(double w, const double *v, const double *rot, double *r)
    {
        M::hoist_row(w, v, rot, r);
    }
    __device__ static double eval(double qx, double qy, double qsq, const double *r)
    {
        return M::eval_row(qx, qy, qsq, r);
    }
};

// ------------------------------------------------------------- rotations ---
// View (theta, phi[, psi]) followed by jitter (dtheta, dphi[, dpsi]) as the
// reverse rotation from detector (qx, qy) to particle (qa, qb, qc).  Same
// matrix products as kernel_iq.c:197-226 and 257-299.

__device__ __forceinline__ void rotation_ac(double theta, double phi,
                                            double dtheta, double dphi,
                                            double *R)
{
    double st, ct, sp, cp;
    sincos(theta*M_PI_180, &st, &ct);
    sincos(phi*M_PI_180, &sp, &cp);
    const double V11 = cp*ct, V12 = sp*ct;
    const double V21 = -sp, V22 = cp;
    const double V31 = st*cp, V32 = sp*st;
    sincos(dtheta*M_PI_180, &st, &ct);
    sincos(dphi*M_PI_180, &sp, &cp);
    const double J31 = st, J32 = -sp*ct, J33 = cp*ct;
    R[0] = J31*V11 + J32*V21 + J33*V31;
    R[1] = J31*V12 + J32*V22 + J33*V32;
}

__device__ __forceinline__ void rotation_abc(double theta, double phi, double psi,
                                             double dtheta, double dphi, double dpsi,
                                             double *R)
{
    double st, ct, sp, cp, ss, cs;
    sincos(theta*M_PI_180, &st, &ct);
    sincos(phi*M_PI_180, &sp, &cp);
    sincos(psi*M_PI_180, &ss, &cs);
    const double V11 = -sp*ss + cp*cs*ct;
    const double V12 = sp*cs*ct + ss*cp;
    const double V21 = -sp*cs - ss*cp*ct;
    const double V22 = -sp*ss*ct + cp*cs;
    const double V31 = st*cp;
    const double V32 = sp*st;
    sincos(dtheta*M_PI_180, &st, &ct);
    sincos(dphi*M_PI_180, &sp, &cp);
    sincos(dpsi*M_PI_180, &ss, &cs);
    const double J11 = cs*ct;
    const double J12 = sp*st*cs + ss*cp;
    const double J13 = sp*ss - st*cp*cs;
    const double J21 = -ss*ct;
    const double J22 = -sp*ss*st + cp*cs;
    const double J23 = sp*cs + ss*st*cp;
    const double J31 = st;
    const double J32 = -sp*ct;
    const double J33 = cp*ct;
    R[0] = J11*V11 + J12*V21 + J13*V31;   // R11
    R[1] = J11*V12 + J12*V22 + J13*V32;   // R12
    R[2] = J21*V11 + J22*V21 + J23*V31;   // R21
    R[3] = J21*V12 + J22*V22 + J23*V32;   // R22
    R[4] = J31*V11 + J32*V21 + J33*V31;   // R31
    R[5] = J31*V12 + J32*V22 + J33*V32;   // R32
}

// ------------------------------------------------------------- magnetism ---
// Spin-resolved cross sections (kernel_iq.c:84-175).  Channel order:
// 0 dd, 1 du.real, 2 ud.real, 3 uu, 4 du.imag, 5 ud.imag.

struct SpinSetup {
    double w[6];
    double cos_mtheta, sin_mtheta, cos_mphi, sin_mphi;
};

__device__ __forceinline__ double clip01(double x)
{
    return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x);
}

// Polarisation-efficiency weights of the six channels.  The normalisation
// makes spin-resolved measurements add up to the (half-)polarised cross
// section: it is the out-going efficiency, or 1 - it when the analyser
// flips the spin (kernel_iq.c:84-124).
__device__ __forceinline__ void spin_setup(const double *values, int npars, SpinSetup &s)
{
    const double in_spin = clip01(values[npars + 2]);
    const double out_spin = clip01(values[npars + 3]);
    const double norm = out_spin < 0.5 ? 1.0 - out_spin : out_spin;
    s.w[0] = (1.0 - in_spin)*(1.0 - out_spin)/norm;
    s.w[1] = (1.0 - in_spin)*out_spin/norm;
    s.w[2] = in_spin*(1.0 - out_spin)/norm;
    s.w[3] = in_spin*out_spin/norm;
    s.w[4] = s.w[1];
    s.w[5] = s.w[2];
    sincos(values[npars + 4]*M_PI_180, &s.sin_mtheta, &s.cos_mtheta);
    sincos(values[npars + 5]*M_PI_180, &s.sin_mphi, &s.cos_mphi);
}

// Effective sld of one magnetic sld in the five distinct channels
// {dd, du.real (= ud.real), uu, du.imag, ud.imag} at detector point (qx, qy).
// M_perp is the magnetisation with its component along q removed; P is the
// polarisation axis and (perpy, perpz) span the plane normal to it.
__device__ __forceinline__ void magnetic_slds(const SpinSetup &s, double qx, double qy,
                                              double sld, double mx, double my, double mz,
                                              double *eff5)
{
    const double qn = sqrt(qx*qx + qy*qy);
    double qhat[3], M[3], P[3], perpy[3], perpz[3], Mperp[3];
    SET_VEC(qhat, qx/qn, qy/qn, 0);
    SET_VEC(M, mx, my, mz);
    SET_VEC(P, s.sin_mtheta*s.cos_mphi, s.sin_mtheta*s.sin_mphi, s.cos_mtheta);
    SET_VEC(perpy, -s.sin_mphi, s.cos_mphi, 0);
    SET_VEC(perpz, -s.cos_mtheta*s.cos_mphi, -s.cos_mtheta*s.sin_mphi, s.sin_mtheta);
    ORTH_VEC(Mperp, M, qhat);
    const double pm = SCALAR_VEC(P, Mperp);
    const double ym = SCALAR_VEC(perpy, Mperp);
    const double zm = SCALAR_VEC(perpz, Mperp);
    eff5[0] = sld - pm;     // dd
    eff5[1] = ym;           // du.real and ud.real
    eff5[2] = sld + pm;     // uu
    eff5[3] = -zm;          // du.imag
    eff5[4] = +zm;          // ud.imag
}

// ------------------------------------------------------ model evaluation ---

template <class M, int XY>
__device__ __forceinline__ double eval_2d(double qx, double qy, double qk,
                                          const double *rot, const double *v)
{
    if constexpr (XY == XY_QA) {
        return M::iq(qk, v);
    } else if constexpr (XY == XY_QAC) {
        // qab^2 = |q|^2 - qc^2 (kernel_iq.c:230-242)
        const double qc = rot[0]*qx + rot[1]*qy;
        const double qab_sq = -qc*qc + qx*qx + qy*qy;
        const double qab = qab_sq > 0.0 ? sqrt(qab_sq) : 0.0;
        return M::iqac(qab, qc, v);
    } else if constexpr (XY == XY_QABC) {
        const double qa = rot[0]*qx + rot[1]*qy;
        const double qb = rot[2]*qx + rot[3]*qy;
        const double qc = rot[4]*qx + rot[5]*qy;
        return M::iqabc(qa, qb, qc, v);
    } else {
        return M::iqxy(qx, qy, v);
    }
}

// ------------------------------------------------------ one mesh point ---

// Decode mesh point `step` (mixed radix over the pd dimensions, weight
// product outermost first, kernel_iq.c:642-664), apply VALID, the jitter
// projection (kernel_iq.c:621-626) and the cutoff, and for a kept point its
// volumes, effective radius and rotation (kernel_iq.c:720-734, 197-312).
// Returns whether the point is kept.
template <class M, int VAR>
__device__ __forceinline__ bool decode_point(
    int step, const DetailsView<M::MAX_PD> &det, const double *__restrict__ values,
    double cutoff, int reff_mode, double *v, double &weight, double &form,
    double &shell, double &reff, double *rot)
{
    using L = Layout<M, VAR>;
    constexpr int MPD = M::MAX_PD;
    #pragma unroll
    for (int k = 0; k < M::NPARS; ++k) v[k] = values[2 + k];
    // Oriented 2D kernels start from zero jitter (kernel_iq.c:614-616, 559).
    if constexpr (L::XY == XY_QAC || L::XY == XY_QABC) {
        if (M::THETA_PAR >= 0) {
            v[M::THETA_PAR] = 0.0;
            v[M::THETA_PAR + 1] = 0.0;
            if (L::XY == XY_QABC) v[M::THETA_PAR + 2] = 0.0;
        }
    }
    const double *pd_value = values + M::NVALUES;
    const double *pd_weight = pd_value + det.num_weights();
    double w = 1.0;
    #pragma unroll
    for (int d = MPD - 1; d >= 0; --d) {
        // lengths and strides were validated on the host; the max() only
        // keeps a malformed buffer from dividing by zero
        const int n = max(det.pd_length(d), 1);
        const int i = (step/max(det.pd_stride(d), 1)) % n;
        const int off = det.pd_offset(d) + i;
        const int p = det.pd_par(d);
        const double pv = pd_value[off];
        #pragma unroll
        for (int k = 0; k < M::NPARS; ++k) if (k == p) v[k] = pv;
        w = pd_weight[off]*w;
    }
    if (!M::valid(v)) return false;
    if constexpr (L::XY == XY_QAC || L::XY == XY_QABC) {
        const double dtheta = v[M::THETA_PAR];
        weight = fabs(cos(dtheta*M_PI_180))*w;     // equirectangular
    } else {
        weight = w;
    }
    if constexpr (L::XY == XY_QXY) {
        // models taking the angles directly see the view angles
        if (M::HAVE_THETA) {
            v[M::THETA_PAR] = values[M::THETA_PAR + 2];
            v[M::THETA_PAR + 1] = values[M::THETA_PAR + 3];
            if (M::HAVE_PSI) v[M::THETA_PAR + 2] = values[M::THETA_PAR + 4];
        }
    }
    if (!(weight > cutoff)) return false;
    M::volume(v, form, shell);
    if (reff_mode != 0) reff = M::reff(reff_mode, v);
    if constexpr (L::XY == XY_QAC) {
        rotation_ac(values[M::THETA_PAR + 2], values[M::THETA_PAR + 3],
                    v[M::THETA_PAR], v[M::THETA_PAR + 1], rot);
    } else if constexpr (L::XY == XY_QABC) {
        rotation_abc(values[M::THETA_PAR + 2], values[M::THETA_PAR + 3],
                     values[M::THETA_PAR + 4], v[M::THETA_PAR],
                     v[M::THETA_PAR + 1], v[M::THETA_PAR + 2], rot);
    }
    return true;
}

// One table row: [weight, p[0..NPARS), rotation] or the binding's hoisted row.
template <class M, int VAR>
__device__ __forceinline__ void write_row(double *row, double weight, const double *v,
                                          const double *rot)
{
    using L = Layout<M, VAR>;
    if constexpr (L::HOISTED) {
        HoistOps<M, true>::row(weight, v, rot, row);
    } else {
        row[0] = weight;
        #pragma unroll
        for (int k = 0; k < M::NPARS; ++k) row[1 + k] = v[k];
        #pragma unroll
        for (int r = 0; r < L::NROT; ++r) row[1 + M::NPARS + r] = rot[r];
    }
}

// ----------------------------------------------------------- mesh_prepare ---

template <class M, int VAR>
__global__ void __launch_bounds__(SEG)
mesh_prepare(int pd_start, int n_mesh, const int32_t *__restrict__ details,
             const double *__restrict__ values, double cutoff, int reff_mode,
             double *__restrict__ table, int *__restrict__ seg_count,
             double *__restrict__ seg_norm, double *__restrict__ points, int points_stride)
{
    using L = Layout<M, VAR>;
    constexpr int NF = L::NF;
    const DetailsView<M::MAX_PD> det{details};
    const int t = threadIdx.x;
    const int local = blockIdx.x*SEG + t;
    const int step = pd_start + local;

    bool keep = false;
    double v[L::NP];
    double weight = 0.0, form = 0.0, shell = 0.0, reff = 0.0;
    double rot[L::NROT > 0 ? L::NROT : 1];

    if (local < n_mesh) {
        keep = decode_point<M, VAR>(step, det, values, cutoff, reff_mode, v, weight, form,
                                    shell, reff, rot);
    }

    // Block-local stable compaction: ballot within warps, prefix over warps.
    __shared__ int warp_base[SEG/32];
    __shared__ double norm_red[4][SEG];
    const int lane = t & 31, warp = t >> 5;
    const unsigned ballot = __ballot_sync(FULL_MASK, keep);
    if (lane == 0) warp_base[warp] = __popc(ballot);
    norm_red[0][t] = keep ? weight : 0.0;
    norm_red[1][t] = keep ? weight*form : 0.0;
    norm_red[2][t] = keep ? weight*shell : 0.0;
    norm_red[3][t] = keep ? weight*reff : 0.0;
    if (points != nullptr && local < n_mesh) {
        // per-point terms of the four norm sums, in mesh order, for the
        // sequential accumulation in finalize (0 for skipped points adds
        // nothing)
        #pragma unroll
        for (int k = 0; k < 4; ++k) points[(size_t)k*points_stride + local] = norm_red[k][t];
    }
    __syncthreads();
    int base = 0, total = 0;
    #pragma unroll
    for (int k = 0; k < SEG/32; ++k) {
        if (k < warp) base += warp_base[k];
        total += warp_base[k];
    }
    if (keep) {
        const int pos = base + __popc(ballot & ((1u << lane) - 1u));
        write_row<M, VAR>(table + ((size_t)blockIdx.x*SEG + pos)*NF, weight, v, rot);
    }
    // fixed-order tree for the four norm sums
    #pragma unroll
    for (int s = SEG/2; s > 0; s >>= 1) {
        __syncthreads();
        if (t < s) {
            #pragma unroll
            for (int k = 0; k < 4; ++k) norm_red[k][t] += norm_red[k][t + s];
        }
    }
    if (t == 0) {
        seg_count[blockIdx.x] = total;
        #pragma unroll
        for (int k = 0; k < 4; ++k) seg_norm[4*blockIdx.x + k] = norm_red[k][0];
    }
}

// ---------------------------------------------------------------- iq_main ---

// Per-lane q point and what depends only on it: |q|, |q|^2 and, for the
// magnetic variant, the effective slds of the five distinct spin channels
// (kernel_iq.c:750-779, hoisted out of the mesh loop).
template <class M, int VAR>
struct QState {
    using L = Layout<M, VAR>;
    static constexpr bool MAG = (VAR == VAR_IMAGNETIC) && (M::NMAG > 0);
    static constexpr int NMAGS = M::NMAG > 0 ? M::NMAG : 1;
    double qk = 0.0, qx = 0.0, qy = 0.0, qsq = 0.0;
    double eff[5][NMAGS];
    double chan_w[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    bool mag_on = false;

    // q is read only for a lane whose q_index is in range (ok): a call with
    // no q points may pass no q array at all
    __device__ __forceinline__ QState(const double *__restrict__ q, int q_index, bool ok,
                                      const double *__restrict__ values)
    {
        if constexpr (L::XY == XY_1D) {
            qk = ok ? q[q_index] : 0.0;
        } else {
            qx = ok ? q[2*q_index] : 0.0;
            qy = ok ? q[2*q_index + 1] : 0.0;
            qsq = qx*qx + qy*qy;
            if constexpr (!L::HOISTED) qk = sqrt(qsq);
        }
        if constexpr (MAG) {
            SpinSetup s;
            spin_setup(values, M::NPARS, s);
            mag_on = (qx*qx + qy*qy) > 1.e-16;
            // channels whose weight is significant (kernel_iq.c:759-761); the
            // two real spin-flip channels see identical slds and share one
            // evaluation
            chan_w[0] = s.w[0] > 1.e-8 ? s.w[0] : 0.0;
            chan_w[1] = (s.w[1] > 1.e-8 ? s.w[1] : 0.0) + (s.w[2] > 1.e-8 ? s.w[2] : 0.0);
            chan_w[2] = s.w[3] > 1.e-8 ? s.w[3] : 0.0;
            chan_w[3] = s.w[4] > 1.e-8 ? s.w[4] : 0.0;
            chan_w[4] = s.w[5] > 1.e-8 ? s.w[5] : 0.0;
            #pragma unroll
            for (int sk = 0; sk < M::NMAG; ++sk) {
                const int idx = M::mag_par(sk);
                const double *m = values + M::NPARS + 6 + 3*sk;
                double e5[5];
                if (mag_on) magnetic_slds(s, qx, qy, values[idx + 2], m[0], m[1], m[2], e5);
                else { e5[0] = e5[1] = e5[2] = e5[3] = e5[4] = 0.0; }
                #pragma unroll
                for (int c = 0; c < 5; ++c) eff[c][sk] = e5[c];
            }
        }
    }
};

// Add w F^2 (and w F) of table rows j0, j0 + step, ... < cnt to acc2 (acc1).
template <class M, int VAR>
__device__ __forceinline__ void accumulate_rows(const QState<M, VAR> &qs,
                                                const double *rows, int j0, int cnt,
                                                int step, double &acc2, double &acc1)
{
    using L = Layout<M, VAR>;
    constexpr int NF = L::NF;
    constexpr int XY = L::XY;
    if constexpr (L::HOISTED) {
        for (int j = j0; j < cnt; j += step)
            acc2 += HoistOps<M, true>::eval(qs.qx, qs.qy, qs.qsq, rows + j*NF);
    } else {
        for (int j = j0; j < cnt; j += step) {
            const double *row = rows + j*NF;
            const double w = row[0];
            double v[L::NP];
            #pragma unroll
            for (int k = 0; k < M::NPARS; ++k) v[k] = row[1 + k];
            const double *rot = row + 1 + M::NPARS;
            if constexpr (XY == XY_1D) {
                if constexpr (L::FQ1D) {
                    double F1, F2;
                    M::fq(qs.qk, F1, F2, v);
                    acc2 += w*F2;
                    acc1 += w*F1;
                } else {
                    acc2 += w*M::iq(qs.qk, v);
                }
            } else if constexpr (QState<M, VAR>::MAG) {
                double F2 = 0.0;
                if (qs.mag_on) {
                    if constexpr (mag_fused<M>::value && XY == XY_QA) {
                        F2 = MagOps<M, true>::channels(qs.qk, v, qs.eff, qs.chan_w);
                    } else {
                        #pragma unroll
                        for (int c = 0; c < 5; ++c) {
                            if (qs.chan_w[c] > 0.0) {
                                #pragma unroll
                                for (int sk = 0; sk < M::NMAG; ++sk)
                                    v[M::mag_par(sk)] = qs.eff[c][sk];
                                F2 += qs.chan_w[c]*eval_2d<M, XY>(qs.qx, qs.qy, qs.qk, rot, v);
                            }
                        }
                    }
                }
                acc2 += w*F2;
            } else {
                acc2 += w*eval_2d<M, XY>(qs.qx, qs.qy, qs.qk, rot, v);
            }
        }
    }
}

// Reduce the per-lane sums of a block to one value per q: butterfly over the
// mesh-lane bits of each warp, then across warps in warp order.  Returns the
// sums in lanes with ml == 0 of warp 0.
template <int LQ, int WARPS, int NOUT>
__device__ __forceinline__ void reduce_block(double &acc2, double &acc1,
                                             double (*red)[LQ][NOUT])
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int qi = lane % LQ;
    const int ml = lane / LQ;
    #pragma unroll
    for (int off = LQ; off < 32; off <<= 1) {
        acc2 += __shfl_xor_sync(FULL_MASK, acc2, off);
        if constexpr (NOUT == 2) acc1 += __shfl_xor_sync(FULL_MASK, acc1, off);
    }
    if (ml == 0) {
        red[warp][qi][0] = acc2;
        if constexpr (NOUT == 2) red[warp][qi][1] = acc1;
    }
    __syncthreads();
    if (warp == 0 && ml == 0) {
        double s2 = 0.0, s1 = 0.0;
        #pragma unroll
        for (int k = 0; k < WARPS; ++k) {
            s2 += red[k][qi][0];
            if constexpr (NOUT == 2) s1 += red[k][qi][1];
        }
        acc2 = s2;
        acc1 = s1;
    }
}

template <class M, int VAR, int LQ, int WARPS>
__global__ void __launch_bounds__(32*WARPS)
iq_main(int nq, const double *__restrict__ q, const double *__restrict__ values,
        const double *__restrict__ table, const int *__restrict__ seg_count,
        int nseg, double *__restrict__ partial)
{
    using L = Layout<M, VAR>;
    constexpr int NF = L::NF;
    constexpr int LM = 32/LQ;

    extern __shared__ __align__(16) double stage[];     // SEG*NF doubles (dynamic)
    __shared__ double red[WARPS][LQ][L::NOUT];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int qi = lane % LQ;
    const int ml = lane / LQ;
    const int q_index = blockIdx.x*LQ + qi;
    const bool q_ok = q_index < nq;
    const QState<M, VAR> qs(q, q_index, q_ok, values);

    const int s0 = (int)(((long long)blockIdx.y*nseg)/gridDim.y);
    const int s1 = (int)(((long long)(blockIdx.y + 1)*nseg)/gridDim.y);
    double acc2 = 0.0, acc1 = 0.0;

    for (int sgi = s0; sgi < s1; ++sgi) {
        const int cnt = seg_count[sgi];
        __syncthreads();
        const double *src = table + (size_t)sgi*SEG*NF;
        for (int i = threadIdx.x; i < cnt*NF; i += 32*WARPS) stage[i] = src[i];
        __syncthreads();
        accumulate_rows<M, VAR>(qs, stage, warp*LM + ml, cnt, WARPS*LM, acc2, acc1);
    }

    reduce_block<LQ, WARPS, L::NOUT>(acc2, acc1, red);
    if (warp == 0 && ml == 0 && q_ok) {
        double *out = partial + (size_t)blockIdx.y*L::NOUT*nq;
        if constexpr (L::FQ1D) {
            out[2*q_index] = acc2;
            out[2*q_index + 1] = acc1;
        } else {
            out[q_index] = acc2;
        }
    }
}

// --------------------------------------------------------------- iq_small ---

// Single-launch form for meshes whose table fits in shared memory
// (n_mesh <= small_mesh_max<M, VAR>()): every block decodes the whole mesh
// range into shared memory (stable compaction in mesh order), evaluates its q
// tile over it and writes -- or, for a continued mesh (accumulate != 0), adds
// to -- its q slots of result directly; block 0 also writes the four norm
// sums.  There is no cross-block reduction, so one launch replaces
// mesh_prepare + iq_main + finalize.  Norms: a fixed tree over the threads'
// strided partial sums, or with an effective radius requested, one point at
// a time in mesh order from the stored value (kernel_iq.c:720-734), as
// finalize does.
template <class M, int VAR>
constexpr int small_mesh_max()
{
    // rows of the table within 32 KB of static shared memory (with the
    // reduction buffers the block stays under the 48 KB static limit), whole
    // warps
    return ((32*1024/(Layout<M, VAR>::NF*8))/32)*32;
}

template <class M, int VAR, int LQ, int WARPS>
__global__ void __launch_bounds__(32*WARPS)
iq_small(int nq, int pd_start, int n_mesh, const int32_t *__restrict__ details,
         const double *__restrict__ values, const double *__restrict__ q, double cutoff,
         int reff_mode, double *__restrict__ result, int accumulate)
{
    using L = Layout<M, VAR>;
    constexpr int NF = L::NF;
    constexpr int LM = 32/LQ;
    constexpr int T = 32*WARPS;
    constexpr int CAP = small_mesh_max<M, VAR>();

    __shared__ __align__(16) double rows[CAP*NF];
    __shared__ double red[WARPS][LQ][L::NOUT];
    __shared__ double nred[4][T];
    __shared__ int warp_cnt[WARPS];

    const DetailsView<M::MAX_PD> det{details};
    const int t = threadIdx.x;
    const int lane = t & 31;
    const int warp = t >> 5;
    const bool norms_here = blockIdx.x == 0;
    const bool sequential = norms_here && reff_mode != 0;

    // ---- the mesh range into shared memory, in mesh order ----
    double nsum[4] = {0.0, 0.0, 0.0, 0.0};
    double seq = 0.0;                        // thread k < 4: norm k in mesh order
    if (sequential && t < 4) seq = accumulate ? result[L::NOUT*nq + t] : 0.0;
    int base = 0;
    for (int chunk = 0; chunk < n_mesh; chunk += T) {
        const int local = chunk + t;
        bool keep = false;
        double v[L::NP];
        double weight = 0.0, form = 0.0, shell = 0.0, reff = 0.0;
        double rot[L::NROT > 0 ? L::NROT : 1];
        if (local < n_mesh)
            keep = decode_point<M, VAR>(pd_start + local, det, values, cutoff, reff_mode, v,
                                        weight, form, shell, reff, rot);
        const double term[4] = {keep ? weight : 0.0, keep ? weight*form : 0.0,
                                keep ? weight*shell : 0.0, keep ? weight*reff : 0.0};
        const unsigned ballot = __ballot_sync(FULL_MASK, keep);
        if (lane == 0) warp_cnt[warp] = __popc(ballot);
        if (sequential) {
            #pragma unroll
            for (int k = 0; k < 4; ++k) nred[k][t] = term[k];
        } else {
            #pragma unroll
            for (int k = 0; k < 4; ++k) nsum[k] += term[k];
        }
        __syncthreads();
        int before = 0, total = 0;
        #pragma unroll
        for (int k = 0; k < WARPS; ++k) {
            if (k < warp) before += warp_cnt[k];
            total += warp_cnt[k];
        }
        if (keep) {
            const int pos = base + before + __popc(ballot & ((1u << lane) - 1u));
            write_row<M, VAR>(rows + pos*NF, weight, v, rot);
        }
        if (sequential && t < 4) {
            const int n = min(T, n_mesh - chunk);
            for (int p = 0; p < n; ++p) seq = __dadd_rn(seq, nred[t][p]);
        }
        base += total;
        __syncthreads();
    }
    const int cnt = base;

    // ---- the norms (block 0) ----
    if (norms_here) {
        if (sequential) {
            if (t < 4) result[L::NOUT*nq + t] = seq;
        } else {
            #pragma unroll
            for (int k = 0; k < 4; ++k) nred[k][t] = nsum[k];
            #pragma unroll
            for (int s = T/2; s > 0; s >>= 1) {
                __syncthreads();
                if (t < s) {
                    #pragma unroll
                    for (int k = 0; k < 4; ++k) nred[k][t] += nred[k][t + s];
                }
            }
            if (t < 4) {
                const double add = nred[t][0];
                result[L::NOUT*nq + t] = accumulate ? result[L::NOUT*nq + t] + add : add;
            }
        }
    }

    // ---- this block's q tile over the table ----
    const int qi = lane % LQ;
    const int ml = lane / LQ;
    const int q_index = blockIdx.x*LQ + qi;
    const bool q_ok = q_index < nq;
    const QState<M, VAR> qs(q, q_index, q_ok, values);
    double acc2 = 0.0, acc1 = 0.0;
    accumulate_rows<M, VAR>(qs, rows, warp*LM + ml, cnt, WARPS*LM, acc2, acc1);
    reduce_block<LQ, WARPS, L::NOUT>(acc2, acc1, red);
    if (warp == 0 && ml == 0 && q_ok) {
        if constexpr (L::FQ1D) {
            result[2*q_index] = accumulate ? result[2*q_index] + acc2 : acc2;
            result[2*q_index + 1] = accumulate ? result[2*q_index + 1] + acc1 : acc1;
        } else {
            result[q_index] = accumulate ? result[q_index] + acc2 : acc2;
        }
    }
}

// --------------------------------------------------------------- finalize ---

// Sum the mesh splits for each output slot in split order, reduce the
// segment norms with a fixed tree in the last block, and store (or add, for
// a call that continues a partly computed mesh) into result.
//
// With `points` (the per-point norm terms of this chunk, in mesh order) the
// four norms are instead accumulated one point at a time from the stored
// value, each add rounded on its own: the order of kernel_iq.c's
// pd_norm/weighted_form/weighted_shell/weighted_radius loop (:720-734), so
// the sums -- and the effective radius and volume ratio derived from them --
// equal the DLL's bit for bit.  run() asks for this when an effective radius
// is requested: P@S feeds these values to S(q), whose closed forms for the
// hard-sphere family cancel to high order at small q R_eff and turn a
// one-ulp difference in R_eff into ~1e-10 in S.
template <int UNUSED = 0>
__global__ void __launch_bounds__(256)
finalize(int nout_nq, int splits, const double *__restrict__ partial,
         int nseg, const double *__restrict__ seg_norm,
         double *__restrict__ result, int accumulate,
         const double *__restrict__ points, int n_points, int points_stride)
{
    if (blockIdx.x + 1 < gridDim.x) {
        const int i = blockIdx.x*256 + threadIdx.x;
        if (i < nout_nq) {
            double s = 0.0;
            for (int k = 0; k < splits; ++k) s += partial[(size_t)k*nout_nq + i];
            result[i] = accumulate ? result[i] + s : s;
        }
        return;
    }
    if (points != nullptr) {
        if (threadIdx.x < 4) {
            const int k = threadIdx.x;
            const double *pk = points + (size_t)k*points_stride;
            double acc = accumulate ? result[nout_nq + k] : 0.0;
            for (int p = 0; p < n_points; ++p) acc = __dadd_rn(acc, pk[p]);
            result[nout_nq + k] = acc;
        }
        return;
    }
    __shared__ double red[4][256];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int sgi = threadIdx.x; sgi < nseg; sgi += 256) {
        #pragma unroll
        for (int k = 0; k < 4; ++k) a[k] += seg_norm[4*sgi + k];
    }
    #pragma unroll
    for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = a[k];
    for (int s = 128; s > 0; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) {
            #pragma unroll
            for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        }
    }
    if (threadIdx.x == 0) {
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            result[nout_nq + k] = accumulate ? result[nout_nq + k] + red[k][0] : red[k][0];
        }
    }
}

}  // namespace sasb200
