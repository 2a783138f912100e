// FP64 core_shell_sphere with the spin channels of the magnetic variant
// sharing one evaluation of the amplitude's q-dependent factors.
//
// Included by the generated translation unit of the core_shell_sphere
// plugin inside its model namespace, after the plugin's own sources, so
// sas_3j1x_x and cube named here are the plugin's (lib/sas_3j1x_x.c,
// kernel_header.c).
//
// The magnetic cross sections (kernel_iq.c:750-779) call the model once per
// significant spin channel with the slds replaced by that channel's
// effective slds.  For core_shell_sphere (core_shell_sphere.c:19-30,
// lib/core_shell.c:8-30) the amplitude is
//
//   f = V_c 3j1(qR)/(qR) (sld_core - sld_shell)
//     + V_s 3j1(q(R+t))/(q(R+t)) (sld_shell - sld_solvent),  F^2 = 1e-4 f f
//
// and only the two contrasts depend on the channel: here the two Bessel
// terms (each a sincos and two divisions) and the two volumes are formed
// once per (q, mesh point) and every channel only recombines them, with the
// reference's operations in the reference's order (V b (contrast) as
// (V b) contrast: the product V b is the same double in every channel).
// 3 j1(x)/x is lib/sas_3j1x_x.c:46-57 restated with its two divisions of
// the closed form as one Newton reciprocal of x (recip_nr, fp64_recip.cuh).
// The non-magnetic variants are the plugin's as translated.

struct SasModelHoisted : SasModel {
    static constexpr bool MAG_FUSED = true;

    // sum over the five distinct channels c with chan_w[c] > 0 of
    // chan_w[c] * F^2(q; v with the slds of channel c); v = radius,
    // thickness, sld_core, sld_shell, sld_solvent
    // 3 j1(x)/x: the reference's series below |x| = 0.1, above it
    // 3 (sin x/x - cos x)/x^2 with r = 1/x as 3 (sin x r - cos x) r^2
    __device__ static double sph_j1x3(double x)
    {
        if (fabs(x) < 0.1) {
            const double x2 = x*x;
            return 1.0 + x2*(-3./30. + x2*(3./840. + x2*(-3./45360.)));
        }
        double s, c;
        sincos(x, &s, &c);
        const double r = recip_nr(x);
        return 3.0*(s*r - c)*(r*r);
    }

    __device__ static double mag_channels(double q, const double *v, const double (*eff)[3],
                                          const double *chan_w)
    {
        const double radius = v[0], thickness = v[1];
        const double vb_core = (M_4PI_3*cube(radius))*sph_j1x3(q*radius);
        const double outer = radius + thickness;
        const double vb_shell = (M_4PI_3*cube(outer))*sph_j1x3(q*outer);
        double F2 = 0.0;
        #pragma unroll
        for (int c = 0; c < 5; ++c) {
            if (chan_w[c] > 0.0) {
                double s[5] = {v[0], v[1], v[2], v[3], v[4]};
                #pragma unroll
                for (int sk = 0; sk < 3; ++sk) s[mag_par(sk)] = eff[c][sk];
                double f = vb_core*(s[2] - s[3]);
                f += vb_shell*(s[3] - s[4]);
                F2 += chan_w[c]*(1.0e-4*f*f);
            }
        }
        return F2;
    }
};
