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
//       [ w * 1e-4 * (drho pi R^2 L)^2,  R,  L/2,  R31,  R32,  0 ]
//     so the contrast, volume, scale factor and weight product are formed
//     once per point instead of once per (q, point);
//   * |q|^2 is formed once per q, and qab^2 = |q|^2 - qc^2;
//   * 2 J1(x)/x on x <= 5 is 2 P(z)/Q(z) (z - Z1)(z - Z2): the reference's
//     J1 = x P/Q (z - Z1)(z - Z2) with the factor x cancelled against the
//     division by x;
//   * on x > 5 the two polynomial ratios share one division, 5/x and the
//     final 1/x share one reciprocal, and 1/sqrt(x) is a reciprocal square
//     root: three divisions and a square root of the reference become two
//     divisions and a reciprocal square root.
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
        row[5] = 0.0;
    }

    // 2 J1(x)/x for x = qab R >= 0
    __device__ static double j1x(double x)
    {
        const double ax = fabs(x);
        if (ax <= 5.0) {
            const double z = ax*ax;
            const double r = polevl(z, RPJ1, 3)/p1evl(z, RQJ1, 8);
            return 2.0*r*(z - Z1)*(z - Z2);
        }
        const double inv = 1.0/ax;
        const double w = 5.0*inv;
        const double z = w*w;
        const double pp = polevl(z, PPJ1, 6), pq = polevl(z, PQJ1, 6);
        const double qp = polevl(z, QPJ1, 7), qq = p1evl(z, QQJ1, 7);
        double sn, cs;
        sincos(ax, &sn, &cs);
        // p (sin - cos) + w q (sin + cos), p = pp/pq, q = qp/qq
        const double num = pp*qq*(sn - cs) + w*qp*pq*(sn + cs);
        return (2.0*SQRT1_PI)*(num/(pq*qq))*inv*rsqrt(ax);
    }

    __device__ static double eval_row(double qx, double qy, double qsq, const double *row)
    {
        const double qc = row[3]*qx + row[4]*qy;
        const double qab_sq = qsq - qc*qc;
        const double qab = qab_sq > 0.0 ? sqrt(qab_sq) : 0.0;
        const double bes = j1x(qab*row[1]);
        const double y = qc*row[2];
        const double sn = y == 0.0 ? 1.0 : sin(y)/y;
        const double f = bes*sn;
        return row[0]*(f*f);
    }
};
