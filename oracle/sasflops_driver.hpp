/*
 * Counting driver for the SAS-flop restatement (measurement infrastructure
 * only).  Included after sasflops.hpp, the reference's model sources and
 * the oracle_* binding written by oracle/build_oracle.py, in a C++
 * translation unit where those sources compute in the counting type SF.
 *
 * It walks the same dispersity mesh as sasmodels/kernel_iq.c:642-714 and
 * evaluates, for every q and every mesh point that passes VALID and the
 * cutoff, the per-evaluation work of kernel_iq.c:737-803 -- the rotation of
 * q into the particle frame (qac/qabc_apply, kernel_iq.c:230-242, 300-312, or
 * |q| for models without orientation), the model call, and the weighted
 * accumulation -- with the reference's own model code, counting its
 * SAS-flops.  Work is reported in three buckets:
 *
 *   eval   per (q, mesh point) evaluation (the metric's unit)
 *   point  once per mesh point: weight product, VALID, jitter projection,
 *          cutoff test, volumes, effective radius, rotation matrix
 *   q      once per q point: the effective magnetic slds of each spin
 *          channel (mag_sld, kernel_iq.c:127-175), which depend only on q
 *          and fixed parameters; the reference evaluates them inside the
 *          mesh loop, an implementation detail that this count hoists
 *
 * and, for the eval bucket, a histogram of the per-evaluation counts (one
 * bin per distinct count: the branch mix).
 */
#undef double
#undef SAS_DOUBLE

#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace sasflops {
thread_local uint64_t count = 0;
}

#define SFL_MAXP (ORACLE_NPARS > 0 ? ORACLE_NPARS : 1)

struct SflPoint {
    SF weight;
    SF v[SFL_MAXP];
    SF rot[6];
};

/* kernel_iq.c:197-226 */
static void sfl_rot_ac(SF theta, SF phi, SF dtheta, SF dphi, SF *R)
{
    SF st, ct, sp, cp;
    SINCOS(theta*M_PI_180, st, ct);
    SINCOS(phi*M_PI_180, sp, cp);
    const SF V11 = cp*ct, V12 = sp*ct, V21 = -sp, V22 = cp;
    const SF V31 = st*cp, V32 = sp*st;
    SINCOS(dtheta*M_PI_180, st, ct);
    SINCOS(dphi*M_PI_180, sp, cp);
    const SF J31 = st, J32 = -sp*ct, J33 = cp*ct;
    R[0] = J31*V11 + J32*V21 + J33*V31;
    R[1] = J31*V12 + J32*V22 + J33*V32;
}

/* kernel_iq.c:257-299 */
static void sfl_rot_abc(SF theta, SF phi, SF psi, SF dtheta, SF dphi, SF dpsi, SF *R)
{
    SF st, ct, sp, cp, ss, cs;
    SINCOS(theta*M_PI_180, st, ct);
    SINCOS(phi*M_PI_180, sp, cp);
    SINCOS(psi*M_PI_180, ss, cs);
    const SF V11 = -sp*ss + cp*cs*ct, V12 = sp*cs*ct + ss*cp;
    const SF V21 = -sp*cs - ss*cp*ct, V22 = -sp*ss*ct + cp*cs;
    const SF V31 = st*cp, V32 = sp*st;
    SINCOS(dtheta*M_PI_180, st, ct);
    SINCOS(dphi*M_PI_180, sp, cp);
    SINCOS(dpsi*M_PI_180, ss, cs);
    const SF J11 = cs*ct, J12 = sp*st*cs + ss*cp, J13 = sp*ss - st*cp*cs;
    const SF J21 = -ss*ct, J22 = -sp*ss*st + cp*cs, J23 = sp*cs + ss*st*cp;
    const SF J31 = st, J32 = -sp*ct, J33 = cp*ct;
    R[0] = J11*V11 + J12*V21 + J13*V31;
    R[1] = J11*V12 + J12*V22 + J13*V32;
    R[2] = J21*V11 + J22*V21 + J23*V31;
    R[3] = J21*V12 + J22*V22 + J23*V32;
    R[4] = J31*V11 + J32*V21 + J33*V31;
    R[5] = J31*V12 + J32*V22 + J33*V32;
}

/* APPLY_ROTATION for one 2D evaluation: qac_apply / qabc_apply
 * (kernel_iq.c:230-242, 300-312); nothing for models without orientation */
static void sfl_apply_rotation(SF qx, SF qy, const SF *rot, SF &qa, SF &qb, SF &qc)
{
#if ORACLE_XY == 2
    const SF dqc = rot[0]*qx + rot[1]*qy;
    const SF dqab_sq = -dqc*dqc + qx*qx + qy*qy;
    qa = dqab_sq > 0.0 ? sqrt(dqab_sq) : SF(0.0);
    qc = dqc;
    (void)qb;
#elif ORACLE_XY == 3
    qa = rot[0]*qx + rot[1]*qy;
    qb = rot[2]*qx + rot[3]*qy;
    qc = rot[4]*qx + rot[5]*qy;
#else
    (void)qx; (void)qy; (void)rot; (void)qa; (void)qb; (void)qc;
#endif
}

/* CALL_KERNEL for one 2D evaluation (kernel_iq.c:522-571): models without
 * orientation take |q| inside the call */
static SF sfl_kernel_2d(SF qx, SF qy, SF qa, SF qb, SF qc, const SF *v)
{
#if ORACLE_XY == 1
    (void)qa; (void)qb; (void)qc;
    return oracle_iq(sqrt(qx*qx + qy*qy), v);
#elif ORACLE_XY == 2
    (void)qx; (void)qy; (void)qb;
    return oracle_iqac(qa, qc, v);
#elif ORACLE_XY == 3
    (void)qx; (void)qy;
    return oracle_iqabc(qa, qb, qc, v);
#else
    (void)qa; (void)qb; (void)qc;
    return oracle_iqxy(qx, qy, v);
#endif
}

#if ORACLE_NMAG > 0
/* kernel_iq.c:127-175 */
static SF sfl_mag_sld(int xs, SF qx, SF qy, SF cos_mt, SF sin_mt, SF cos_mp, SF sin_mp,
                      SF sld, SF mx, SF my, SF mz)
{
    SF M[3], P[3], qv[3], py[3], pz[3], Mp[3];
    const SF qn = sqrt(qx*qx + qy*qy);
    SET_VEC(qv, qx/qn, qy/qn, SF(0.0));
    SET_VEC(M, mx, my, mz);
    SET_VEC(P, sin_mt*cos_mp, sin_mt*sin_mp, cos_mt);
    SET_VEC(py, -sin_mp, cos_mp, SF(0.0));
    SET_VEC(pz, -cos_mt*cos_mp, -cos_mt*sin_mp, sin_mt);
    ORTH_VEC(Mp, M, qv);
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
 * variant: 0 = 1D, 1 = 2D, 2 = 2D magnetic.  totals[0..4] = eval SAS-flops,
 * point SAS-flops, q SAS-flops, evaluations, kept mesh points.  hist[c] =
 * number of evaluations that cost c SAS-flops (c < nbins - 1; the last bin
 * collects the rest).  Returns 0, -1 for a magnetic call of a model without
 * slds.
 */
extern "C" int sasflops_count(int variant, int32_t nq, const int32_t *details,
                              const double *values_in, int32_t nvalues, const double *q,
                              double cutoff_in, int32_t reff_mode, int threads,
                              uint64_t *totals, uint64_t *hist, int32_t nbins)
{
    const int MPD = ORACLE_MAX_PD;
    const int xy = variant == 0 ? 0 : ORACLE_XY;
    const int fq1d = variant == 0 && ORACLE_HAVE_FQ;
    if (variant == 2 && ORACLE_NMAG == 0) return -1;
    std::vector<SF> values(values_in, values_in + nvalues);
    const SF cutoff(cutoff_in);
    const int32_t *pd_par = details, *pd_length = details + MPD;
    const int32_t *pd_offset = details + 2*MPD, *pd_stride = details + 3*MPD;
    const int num_eval = details[4*MPD];
    const int num_weights = details[4*MPD + 1];
    const SF *pd_value = values.data() + ORACLE_NVALUES;
    const SF *pd_weight = pd_value + num_weights;
    for (int k = 0; k < 5; ++k) totals[k] = 0;
    for (int k = 0; k < nbins; ++k) hist[k] = 0;

    /* ---- mesh walk (point bucket) ---- */
    std::vector<SflPoint> mesh;
    mesh.reserve(num_eval > 0 ? num_eval : 1);
    SF norm[4] = {SF(0.0), SF(0.0), SF(0.0), SF(0.0)};
    sasflops::count = 0;
    for (int step = 0; step < num_eval; ++step) {
        SF v[SFL_MAXP];
        for (int k = 0; k < ORACLE_NPARS; ++k) v[k] = values[2 + k];
#if ORACLE_THETA_PAR >= 0
        if (xy == 2 || xy == 3) {
            v[ORACLE_THETA_PAR] = 0.0;
            v[ORACLE_THETA_PAR + 1] = 0.0;
            if (xy == 3) v[ORACLE_THETA_PAR + 2] = 0.0;
        }
#endif
        SF w(1.0);
        for (int d = MPD - 1; d >= 0; --d) {
            const int i = (step/pd_stride[d]) % pd_length[d];
            v[pd_par[d]] = pd_value[pd_offset[d] + i];
            w = pd_weight[pd_offset[d] + i]*w;
        }
        if (!oracle_valid(v)) continue;
        SF weight = w;
#if ORACLE_THETA_PAR >= 0
        if (xy == 2 || xy == 3) weight = fabs(cos(v[ORACLE_THETA_PAR]*M_PI_180))*w;
        if (xy == 4 && ORACLE_HAVE_THETA) {
            v[ORACLE_THETA_PAR] = values[ORACLE_THETA_PAR + 2];
            v[ORACLE_THETA_PAR + 1] = values[ORACLE_THETA_PAR + 3];
            if (ORACLE_HAVE_PSI) v[ORACLE_THETA_PAR + 2] = values[ORACLE_THETA_PAR + 4];
        }
#endif
        if (!(weight > cutoff)) continue;
        SF form, shell;
        oracle_volume(v, &form, &shell);
        norm[0] += weight;
        norm[1] += weight*form;
        norm[2] += weight*shell;
        if (reff_mode != 0) norm[3] += weight*oracle_reff(reff_mode, v);
        SflPoint p;
        p.weight = weight;
        for (int k = 0; k < SFL_MAXP; ++k) p.v[k] = v[k];
#if ORACLE_THETA_PAR >= 0
        if (xy == 2) {
            sfl_rot_ac(values[ORACLE_THETA_PAR + 2], values[ORACLE_THETA_PAR + 3],
                       v[ORACLE_THETA_PAR], v[ORACLE_THETA_PAR + 1], p.rot);
        } else if (xy == 3) {
            sfl_rot_abc(values[ORACLE_THETA_PAR + 2], values[ORACLE_THETA_PAR + 3],
                        values[ORACLE_THETA_PAR + 4], v[ORACLE_THETA_PAR],
                        v[ORACLE_THETA_PAR + 1], v[ORACLE_THETA_PAR + 2], p.rot);
        }
#endif
        mesh.push_back(p);
    }
    totals[1] = sasflops::count;
    totals[4] = mesh.size();
    const int n_kept = (int)mesh.size();

#if ORACLE_NMAG > 0
    SF xs_w[6], cos_mt(0.0), sin_mt(0.0), cos_mp(0.0), sin_mp(0.0);
    if (variant == 2) {
        /* kernel_iq.c:84-124, once per call */
        SF in_spin = clip(values[ORACLE_NPARS + 2], SF(0.0), SF(1.0));
        SF out_spin = clip(values[ORACLE_NPARS + 3], SF(0.0), SF(1.0));
        const SF nrm = out_spin < 0.5 ? SF(1.0) - out_spin : out_spin;
        xs_w[0] = (SF(1.0) - in_spin)*(SF(1.0) - out_spin)/nrm;
        xs_w[1] = (SF(1.0) - in_spin)*out_spin/nrm;
        xs_w[2] = in_spin*(SF(1.0) - out_spin)/nrm;
        xs_w[3] = in_spin*out_spin/nrm;
        xs_w[4] = xs_w[1];
        xs_w[5] = xs_w[2];
        SINCOS(values[ORACLE_NPARS + 4]*M_PI_180, sin_mt, cos_mt);
        SINCOS(values[ORACLE_NPARS + 5]*M_PI_180, sin_mp, cos_mp);
    }
#endif

    /* ---- per-q evaluations (eval and q buckets) ---- */
    uint64_t eval_total = 0, q_total = 0, evals = 0;
#ifdef _OPENMP
    #pragma omp parallel num_threads(threads > 0 ? threads : 1) \
        reduction(+:eval_total, q_total, evals)
#endif
    {
        std::vector<uint64_t> h(nbins, 0);
#ifdef _OPENMP
        #pragma omp for schedule(dynamic, 4)
#endif
        for (int qi = 0; qi < nq; ++qi) {
            SF qk(0.0), qx(0.0), qy(0.0);
            if (xy == 0) qk = q[qi];
            else { qx = q[2*qi]; qy = q[2*qi + 1]; }
#if ORACLE_NMAG > 0
            SF eff[6][ORACLE_NMAG];
            if (variant == 2) {
                sasflops::count = 0;
                if ((double)qx*(double)qx + (double)qy*(double)qy > 1.e-16) {
                    for (int xs = 0; xs < 6; ++xs) {
                        if (!((double)xs_w[xs] > 1.e-8)) continue;
                        for (int sk = 0; sk < ORACLE_NMAG; ++sk) {
                            const int idx = oracle_mag_par(sk);
                            const SF *mm = values.data() + ORACLE_NPARS + 6 + 3*sk;
                            eff[xs][sk] = sfl_mag_sld(xs, qx, qy, cos_mt, sin_mt, cos_mp,
                                                      sin_mp, values[idx + 2],
                                                      mm[0], mm[1], mm[2]);
                        }
                    }
                }
                q_total += sasflops::count;
            }
#endif
            SF acc2(0.0), acc1(0.0);
            for (int m = 0; m < n_kept; ++m) {
                const SflPoint &p = mesh[m];
                SF v[SFL_MAXP];
                for (int k = 0; k < SFL_MAXP; ++k) v[k] = p.v[k];
                sasflops::count = 0;
                SF F1(0.0), F2(0.0);
                if (xy == 0) {
                    if (fq1d) oracle_fq(qk, &F1, &F2, v);
                    else F2 = oracle_iq(qk, v);
                } else {
                    SF qa(0.0), qb(0.0), qc(0.0);
                    sfl_apply_rotation(qx, qy, p.rot, qa, qb, qc);
                    if (variant == 2) {
#if ORACLE_NMAG > 0
                        const SF qsq = qx*qx + qy*qy;
                        if (qsq > 1.e-16) {
                            for (int xs = 0; xs < 6; ++xs) {
                                if (xs_w[xs] > 1.e-8) {
                                    for (int sk = 0; sk < ORACLE_NMAG; ++sk)
                                        v[oracle_mag_par(sk)] = eff[xs][sk];
                                    F2 += xs_w[xs]*sfl_kernel_2d(qx, qy, qa, qb, qc, v);
                                }
                            }
                        }
#endif
                    } else {
                        F2 = sfl_kernel_2d(qx, qy, qa, qb, qc, v);
                    }
                }
                acc2 += p.weight*F2;
                if (fq1d) acc1 += p.weight*F1;
                const uint64_t c = sasflops::count;
                eval_total += c;
                ++evals;
                ++h[c < (uint64_t)(nbins - 1) ? c : (uint64_t)(nbins - 1)];
            }
        }
#ifdef _OPENMP
        #pragma omp critical
#endif
        for (int k = 0; k < nbins; ++k) hist[k] += h[k];
    }
    totals[0] = eval_total;
    totals[2] = q_total;
    totals[3] = evals;
    (void)norm;
    return 0;
}
