// FP64 cylinder 2D with the per-mesh-point work hoisted out of the q loop.
//
// Included by the generated translation unit of the cylinder plugin inside
// its model namespace, after the plugin's own sources, so the J1 tables
// (RPJ1 ... QQJ1 of lib/sas_J1.c) and polevl/p1evl (lib/polevl.c) named
// here are the plugin's.
//
// The quantity is the reference's, cylinder.c:92-102 (Iqac), :7-11 (_fq),
// lib/sas_J1.c:107-153 and :240-245 (cephes_j1, sas_2J1x_x), with
// kernel_iq.c:230-242 (qac_apply) and :789-803 (the weighted accumulation):
//
//   w * 1e-4 * (drho * pi R^2 L * 2 J1(qab R)/(qab R) * sin(qc L/2)/(qc L/2))^2
//
// Arithmetic is rearranged, not approximated differently:
//
//   * mesh_prepare stores per kept mesh point the row
//       [ w * 1e-4 * (drho pi R^2 L)^2,  R,  L/2,  R31,  R32,  R^2 ]
//     so the contrast, volume, scale factor and weight product are formed
//     once per point instead of once per (q, point);
//   * |q|^2 is formed once per q, and qab^2 = |q|^2 - qc^2;
//   * 2 J1(x)/x on x <= 5 is 2 P(z)/Q(z) (z - Z1)(z - Z2) with z = x^2 =
//     qab^2 R^2: the reference's J1 = x P/Q (z - Z1)(z - Z2) with the
//     factor x cancelled against the division by x, and no square root for
//     qab on this branch (about four evaluations in five);
//   * on x > 5 the two polynomial ratios share one division, 5/x and the
//     final 1/x share one reciprocal, and 1/sqrt(x) is a reciprocal square
//     root;
//   * sin(y)/y of the length factor joins the J1 term's division, so an
//     evaluation divides once on x <= 5 and twice on x > 5 (the reference:
//     three and five times);
//   * those divisions are a multiplication by a reciprocal from Newton's
//     method (recip_nr, fp64_recip.cuh), within an ulp or two of 1/d.  Its
//     arguments stay in the normal range: den is a positive polynomial
//     value, x > 5 on the asymptotic branch, and |y| < 1e-100 counts as
//     y = 0, where sin(y)/y already rounds to 1.
//
// Each change moves a result by a few units in the last place; the mesh
// sums of these non-negative terms stay within 1e-12 of the reference DLL
// (the parity tests' bar).

struct SasModelHoisted : SasModel {
    static constexpr int HOIST = 2;     // the qac (oriented, symmetric) form
    static constexpr int NH = 6;

    // squares of the first two zeros of J1, and 1/sqrt(pi)
    static constexpr double Z1 = 1.46819706421238932572E1;
    static constexpr double Z2 = 4.92184563216946036703E1;
    static constexpr double SQRT1_PI = 0.56418958354775628;

    // v = sld, sld_solvent, radius, length, theta, phi; rot = R31, R32
    __device__ static void hoist_row(double weight, const double *v, const double *rot,
                                     double *row)
    {
        const double s = (v[0] - v[1])*form_volume(v[2], v[3]);
        row[0] = weight*(1.0e-4*(s*s));
        row[1] = v[2];
        row[2] = 0.5*v[3];
        row[3] = rot[0];
        row[4] = rot[1];
        row[5] = v[2]*v[2];
    }

    // two consecutive doubles of a 16-byte aligned row in one shared load
    __device__ static void pair(const double *p, double &a, double &b)
    {
#ifdef __CUDA_ARCH__
        const double2 t = *reinterpret_cast<const double2 *>(p);
        a = t.x;
        b = t.y;
#else
        a = p[0];
        b = p[1];
#endif
    }

    // 2 J1(x)/x as num/den, for x^2 = z (x = qab R >= 0; qab_sq = qab^2)
    __device__ static void j1x_parts(double z, double qab_sq, double R, double &num,
                                     double &den)
    {
        if (z <= 25.0) {
            num = 2.0*polevl(z, RPJ1, 3)*(z - Z1)*(z - Z2);
            den = p1evl(z, RQJ1, 8);
            return;
        }
        const double ax = sqrt(qab_sq)*R;
        const double inv = recip_nr(ax);
        const double w = 5.0*inv;
        const double zz = w*w;
        const double pp = polevl(zz, PPJ1, 6), pq = polevl(zz, PQJ1, 6);
        const double qp = polevl(zz, QPJ1, 7), qq = p1evl(zz, QQJ1, 7);
        double sn, cs;
        sincos(ax, &sn, &cs);
        // p (sin - cos) + w q (sin + cos), p = pp/pq, q = qp/qq
        num = (pp*qq*(sn - cs) + w*qp*pq*(sn + cs))*((2.0*SQRT1_PI)*inv*rsqrt(ax));
        den = pq*qq;
    }

    // 2 J1(x)/x for x >= 0 (used by the host checks)
    __device__ static double j1x(double x)
    {
        double num, den;
        j1x_parts(x*x, x*x, 1.0, num, den);
        return num/den;
    }

    __device__ static double eval_row(double qx, double qy, double qsq, const double *row)
    {
        double A, R, halfL, R31, R32, R2;
        pair(row, A, R);
        pair(row + 2, halfL, R31);
        pair(row + 4, R32, R2);
        const double qc = R31*qx + R32*qy;
        const double qab_sq = qsq - qc*qc;
        const double z = qab_sq > 0.0 ? qab_sq*R2 : 0.0;
        double num, den;
        j1x_parts(z, qab_sq, R, num, den);
        // sin(y)/y folded into the same division (1 at y = 0)
        const double y = qc*halfL;
        const bool y0 = fabs(y) < 1.0e-100;
        const double f = (num*(y0 ? 1.0 : sin(y)))*recip_nr(den*(y0 ? 1.0 : y));
        return A*(f*f);
    }
};
