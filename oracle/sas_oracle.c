/*
 * CPU restatement of the sasmodels kernel driver (test infrastructure only:
 * the checker for the B200 kernels, never the product path).
 *
 * Restates sasmodels/kernel_iq.c:317-847 for one model whose functions are
 * bound by the including translation unit through the ORACLE_* macros and
 * oracle_* functions (written by oracle/build_oracle.py).  Same arithmetic,
 * same order per q point:
 *
 *   phase 1 (serial): walk the dispersity mesh [pd_start, pd_stop) in the
 *     reference's loop order (kernel_iq.c:642-714), forming the weight
 *     product outermost-first, the parameter vector, VALID, the jitter
 *     projection (kernel_iq.c:621-626) and the cutoff, accumulating the four
 *     norms (kernel_iq.c:726-734) and the per-point rotation
 *     (kernel_iq.c:197-312);
 *   phase 2 (OpenMP over q): for each q, accumulate w*F^2 (and w*F) over the
 *     surviving points in mesh order (kernel_iq.c:737-803), with the
 *     magnetic cross sections of kernel_iq.c:750-779.
 *
 * Because each q sums in mesh order exactly as the reference DLL does, the
 * result is bitwise the DLL's when compiled with the same flags, at any
 * thread count (the reference's own OpenMP mode shares loop variables across
 * threads and is not used).
 */
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXP (ORACLE_NPARS > 0 ? ORACLE_NPARS : 1)
#define NROT (ORACLE_XY == 2 ? 2 : (ORACLE_XY == 3 ? 6 : 0))

typedef struct {
    double weight;
    double v[MAXP];
    double rot[6];
} MeshPoint;

/* kernel_iq.c:197-226 */
static void oracle_rot_ac(double theta, double phi, double dtheta, double dphi, double *R)
{
    double st, ct, sp, cp;
    SINCOS(theta*M_PI_180, st, ct);
    SINCOS(phi*M_PI_180, sp, cp);
    const double V11 = cp*ct, V12 = sp*ct, V21 = -sp, V22 = cp;
    const double V31 = st*cp, V32 = sp*st;
    SINCOS(dtheta*M_PI_180, st, ct);
    SINCOS(dphi*M_PI_180, sp, cp);
    const double J31 = st, J32 = -sp*ct, J33 = cp*ct;
    R[0] = J31*V11 + J32*V21 + J33*V31;
    R[1] = J31*V12 + J32*V22 + J33*V32;
}

/* kernel_iq.c:257-299 */
static void oracle_rot_abc(double theta, double phi, double psi,
                           double dtheta, double dphi, double dpsi, double *R)
{
    double st, ct, sp, cp, ss, cs;
    SINCOS(theta*M_PI_180, st, ct);
    SINCOS(phi*M_PI_180, sp, cp);
    SINCOS(psi*M_PI_180, ss, cs);
    const double V11 = -sp*ss + cp*cs*ct;
    const double V12 = sp*cs*ct + ss*cp;
    const double V21 = -sp*cs - ss*cp*ct;
    const double V22 = -sp*ss*ct + cp*cs;
    const double V31 = st*cp;
    const double V32 = sp*st;
    SINCOS(dtheta*M_PI_180, st, ct);
    SINCOS(dphi*M_PI_180, sp, cp);
    SINCOS(dpsi*M_PI_180, ss, cs);
    const double J11 = cs*ct;
    const double J12 = sp*st*cs + ss*cp;
    const double J13 = sp*ss - st*cp*cs;
    const double J21 = -ss*ct;
    const double J22 = -sp*ss*st + cp*cs;
    const double J23 = sp*cs + ss*st*cp;
    const double J31 = st;
    const double J32 = -sp*ct;
    const double J33 = cp*ct;
    R[0] = J11*V11 + J12*V21 + J13*V31;
    R[1] = J11*V12 + J12*V22 + J13*V32;
    R[2] = J21*V11 + J22*V21 + J23*V31;
    R[3] = J21*V12 + J22*V22 + J23*V32;
    R[4] = J31*V11 + J32*V21 + J33*V31;
    R[5] = J31*V12 + J32*V22 + J33*V32;
}

/* 2D model call for the model's orientation mode (kernel_iq.c:531-571) */
static double oracle_call_2d(double qx, double qy, const double *rot, const double *v)
{
#if ORACLE_XY == 1
    (void)rot;
    return oracle_iq(sqrt(qx*qx + qy*qy), v);
#elif ORACLE_XY == 2
    const double qc = rot[0]*qx + rot[1]*qy;
    const double qab_sq = -qc*qc + qx*qx + qy*qy;
    const double qab = qab_sq > 0.0 ? sqrt(qab_sq) : 0.0;
    return oracle_iqac(qab, qc, v);
#elif ORACLE_XY == 3
    const double qa = rot[0]*qx + rot[1]*qy;
    const double qb = rot[2]*qx + rot[3]*qy;
    const double qc = rot[4]*qx + rot[5]*qy;
    return oracle_iqabc(qa, qb, qc, v);
#else
    (void)rot;
    return oracle_iqxy(qx, qy, v);
#endif
}

#if ORACLE_NMAG > 0
/* kernel_iq.c:84-124 */
static void oracle_spin_weights(double in_spin, double out_spin, double w[6])
{
    in_spin = clip(in_spin, 0.0, 1.0);
    out_spin = clip(out_spin, 0.0, 1.0);
    const double norm = out_spin < 0.5 ? 1 - out_spin : out_spin;
    w[0] = (1.0 - in_spin)*(1.0 - out_spin)/norm;
    w[1] = (1.0 - in_spin)*out_spin/norm;
    w[2] = in_spin*(1.0 - out_spin)/norm;
    w[3] = in_spin*out_spin/norm;
    w[4] = w[1];
    w[5] = w[2];
}

/* kernel_iq.c:127-175 */
static double oracle_mag_sld(int xs, double qx, double qy, double cos_mt, double sin_mt,
                             double cos_mp, double sin_mp, double sld,
                             double mx, double my, double mz)
{
    double M[3], P[3], q[3], py[3], pz[3], Mp[3];
    const double qn = sqrt(qx*qx + qy*qy);
    SET_VEC(q, qx/qn, qy/qn, 0);
    SET_VEC(M, mx, my, mz);
    SET_VEC(P, sin_mt*cos_mp, sin_mt*sin_mp, cos_mt);
    SET_VEC(py, -sin_mp, cos_mp, 0);
    SET_VEC(pz, -cos_mt*cos_mp, -cos_mt*sin_mp, sin_mt);
    ORTH_VEC(Mp, M, q);
    switch (xs) {
    case 0: return sld - SCALAR_VEC(P, Mp);
    case 1: case 2: return SCALAR_VEC(py, Mp);
    case 3: return sld + SCALAR_VEC(P, Mp);
    case 4: return -SCALAR_VEC(pz, Mp);
    default: return +SCALAR_VEC(pz, Mp);
    }
}
#endif

/*
 * variant: 0 = 1D (Iq), 1 = 2D (Iqxy), 2 = 2D magnetic (Imagnetic).
 * result: nout*nq + 4 doubles, nout = 2 for 1D Fq models.
 * Returns 0, or -1 if the magnetic variant is asked of a model without slds,
 * -2 on allocation failure.
 */
int oracle_kernel(int variant, int32_t nq, int32_t pd_start, int32_t pd_stop,
                  const int32_t *details, const double *values, const double *q,
                  double *result, double cutoff, int32_t reff_mode, int threads)
{
    const int MPD = ORACLE_MAX_PD;
    const int xy = variant == 0 ? 0 : ORACLE_XY;
    const int fq1d = variant == 0 && ORACLE_HAVE_FQ;
    const int nout = fq1d ? 2 : 1;
    if (variant == 2 && ORACLE_NMAG == 0) return -1;
    const int32_t *pd_par = details, *pd_length = details + MPD;
    const int32_t *pd_offset = details + 2*MPD, *pd_stride = details + 3*MPD;
    const int num_weights = details[4*MPD + 1];
    const double *pd_value = values + ORACLE_NVALUES;
    const double *pd_weight = pd_value + num_weights;

    double norm[4];
    for (int k = 0; k < 4; ++k) norm[k] = pd_start == 0 ? 0.0 : result[nout*nq + k];
    if (pd_start == 0) memset(result, 0, sizeof(double)*nout*nq);

    const int n_mesh = pd_stop - pd_start;
    MeshPoint *mesh = (MeshPoint *)malloc(sizeof(MeshPoint)*(n_mesh > 0 ? n_mesh : 1));
    if (!mesh) return -2;
    int n_kept = 0;

    /* ---- phase 1: mesh walk ---- */
    for (int step = pd_start; step < pd_stop; ++step) {
        double v[MAXP];
        for (int k = 0; k < ORACLE_NPARS; ++k) v[k] = values[2 + k];
#if ORACLE_THETA_PAR >= 0
        if (xy == 2 || xy == 3) {
            v[ORACLE_THETA_PAR] = 0.0;
            v[ORACLE_THETA_PAR + 1] = 0.0;
            if (xy == 3) v[ORACLE_THETA_PAR + 2] = 0.0;
        }
#endif
        double w = 1.0;
        for (int d = MPD - 1; d >= 0; --d) {
            const int i = (step/pd_stride[d]) % pd_length[d];
            v[pd_par[d]] = pd_value[pd_offset[d] + i];
            w = pd_weight[pd_offset[d] + i]*w;
        }
        if (!oracle_valid(v)) continue;
        double weight = w;
#if ORACLE_THETA_PAR >= 0
        if (xy == 2 || xy == 3) weight = fabs(cos(v[ORACLE_THETA_PAR]*M_PI_180))*w;
        if (xy == 4 && ORACLE_HAVE_THETA) {
            v[ORACLE_THETA_PAR] = values[ORACLE_THETA_PAR + 2];
            v[ORACLE_THETA_PAR + 1] = values[ORACLE_THETA_PAR + 3];
            if (ORACLE_HAVE_PSI) v[ORACLE_THETA_PAR + 2] = values[ORACLE_THETA_PAR + 4];
        }
#endif
        if (!(weight > cutoff)) continue;
        double form, shell;
        oracle_volume(v, &form, &shell);
        norm[0] += weight;
        norm[1] += weight*form;
        norm[2] += weight*shell;
        if (reff_mode != 0) norm[3] += weight*oracle_reff(reff_mode, v);
        MeshPoint *p = &mesh[n_kept++];
        p->weight = weight;
        memcpy(p->v, v, sizeof(v));
#if ORACLE_THETA_PAR >= 0
        if (xy == 2) {
            oracle_rot_ac(values[ORACLE_THETA_PAR + 2], values[ORACLE_THETA_PAR + 3],
                          v[ORACLE_THETA_PAR], v[ORACLE_THETA_PAR + 1], p->rot);
        } else if (xy == 3) {
            oracle_rot_abc(values[ORACLE_THETA_PAR + 2], values[ORACLE_THETA_PAR + 3],
                           values[ORACLE_THETA_PAR + 4], v[ORACLE_THETA_PAR],
                           v[ORACLE_THETA_PAR + 1], v[ORACLE_THETA_PAR + 2], p->rot);
        }
#endif
    }

#if ORACLE_NMAG > 0
    double xs_w[6], cos_mt, sin_mt, cos_mp, sin_mp;
    if (variant == 2) {
        oracle_spin_weights(values[ORACLE_NPARS + 2], values[ORACLE_NPARS + 3], xs_w);
        SINCOS(values[ORACLE_NPARS + 4]*M_PI_180, sin_mt, cos_mt);
        SINCOS(values[ORACLE_NPARS + 5]*M_PI_180, sin_mp, cos_mp);
    }
#endif

    /* ---- phase 2: per-q sums in mesh order ---- */
#ifdef _OPENMP
    #pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
#else
    (void)threads;
#endif
    for (int qi = 0; qi < nq; ++qi) {
        double acc2 = result[nout*qi], acc1 = fq1d ? result[nout*qi + 1] : 0.0;
        double qk = 0.0, qx = 0.0, qy = 0.0;
        if (xy == 0) qk = q[qi];
        else { qx = q[2*qi]; qy = q[2*qi + 1]; }
        for (int m = 0; m < n_kept; ++m) {
            const MeshPoint *p = &mesh[m];
            double v[MAXP];
            memcpy(v, p->v, sizeof(v));
            double F1 = 0.0, F2;
            if (xy == 0) {
                if (fq1d) oracle_fq(qk, &F1, &F2, v);
                else F2 = oracle_iq(qk, v);
            } else if (variant == 2) {
                F2 = 0.0;
#if ORACLE_NMAG > 0
                if (qx*qx + qy*qy > 1.e-16) {
                    for (int xs = 0; xs < 6; ++xs) {
                        if (xs_w[xs] > 1.e-8) {
                            for (int sk = 0; sk < ORACLE_NMAG; ++sk) {
                                const int idx = oracle_mag_par(sk);
                                const double *mm = values + ORACLE_NPARS + 6 + 3*sk;
                                v[idx] = oracle_mag_sld(xs, qx, qy, cos_mt, sin_mt, cos_mp,
                                                        sin_mp, values[idx + 2],
                                                        mm[0], mm[1], mm[2]);
                            }
                            F2 += xs_w[xs]*oracle_call_2d(qx, qy, p->rot, v);
                        }
                    }
                }
#endif
            } else {
                F2 = oracle_call_2d(qx, qy, p->rot, v);
            }
            acc2 += p->weight*F2;
            if (fq1d) acc1 += p->weight*F1;
        }
        result[nout*qi] = acc2;
        if (fq1d) result[nout*qi + 1] = acc1;
    }
    for (int k = 0; k < 4; ++k) result[nout*nq + k] = norm[k];
    free(mesh);
    return 0;
}
