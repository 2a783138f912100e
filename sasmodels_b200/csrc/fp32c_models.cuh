// FP32-compensated physics of the measured models.
//
// The amplitudes restate the model plugins' formulas with FP32 bulk
// arithmetic (fp32c_math.cuh), FP64 phases, and FP64 orientation/shape
// quadrature sums; volumes, validity and effective radii keep using the
// plugin's own FP64 functions (the binding struct inherits them).
//
//   sphere               sphere.c:13-20
//   cylinder             cylinder.c:7-11, 55-102
//   core_shell_sphere    core_shell_sphere.c:19-30, lib/core_shell.c:8-30
//   ellipsoid            ellipsoid.c:50-105
//   core_shell_cylinder  core_shell_cylinder.c:4-7, 60-123
//
// The adaptive Gauss-Legendre order follows lib/adaptive.c:11290-11297
// (20/76/500/5000 points for q*r_max < 10/100/750/else), evaluated in FP64
// so the FP32c form picks the same rule as the FP64 form.  Rule tables are
// the plugin's own nodes and weights (copied by the generator into global
// memory next to FP64 sin/cos of the cylinder angle for each node).
#pragma once

#include "fp32c_math.cuh"

namespace f32c {

struct Rule {
    int n;
    const double *z, *w, *st, *ct;
};

// Defined by the generated translation unit (needs the plugin's tables).
__device__ __forceinline__ Rule rule_for(double qr);

constexpr double PI_4 = 0.7853981633974483;     // kernel_header.c M_PI_4
constexpr double PI = 3.141592653589793;
constexpr double FOUR_PI_3 = 4.18879020478639;  // kernel_header.c M_4PI_3

// ---- sphere ---------------------------------------------------------------
__device__ __forceinline__ void sphere_fq(double q, double sld, double solvent,
                                         double radius, double &F1, double &F2)
{
    const double bes = (double)sph_j1c_f(q*radius);
    const double form = (sld - solvent)*(FOUR_PI_3*radius*radius*radius)*bes;
    F1 = 1.0e-2*form;
    F2 = 1.0e-4*form*form;
}

// ---- core_shell_sphere ----------------------------------------------------
__device__ __forceinline__ void core_shell_sphere_fq(double q, double radius, double thickness,
                                                     double core_sld, double shell_sld,
                                                     double solvent_sld, double &F1, double &F2)
{
    const double rt = radius + thickness;
    const float core = (float)(FOUR_PI_3*radius*radius*radius*(core_sld - shell_sld));
    const float shell = (float)(FOUR_PI_3*rt*rt*rt*(shell_sld - solvent_sld));
    const float f = core*sph_j1c_f(q*radius) + shell*sph_j1c_f(q*rt);
    F1 = 1.0e-2*(double)f;
    F2 = 1.0e-4*(double)f*(double)f;
}

// ---- cylinder ---------------------------------------------------------------
__device__ __forceinline__ double cylinder_iqac(double qab, double qc, double sld,
                                                double solvent, double radius, double length)
{
    const float form = j1c_f(qab*radius)*sinc_f(qc*0.5*length);
    const double s = (sld - solvent)*(PI*radius*radius*length);
    const double a = s*(double)form;
    return 1.0e-4*a*a;
}

__device__ __forceinline__ void cylinder_fq(double q, double sld, double solvent,
                                            double radius, double length,
                                            double &F1, double &F2)
{
    const Rule r = rule_for(q*fmax(radius, 0.5*length));
    const double qr = q*radius, qh = q*0.5*length;
    double t1 = 0.0, t2 = 0.0;
    for (int i = 0; i < r.n; ++i) {
        const double st = r.st[i], ct = r.ct[i];
        const float form = j1c_f(qr*st)*sinc_f(qh*ct);
        const double wf = r.w[i]*st*(double)form;
        t1 += wf;
        t2 = fma(wf, (double)form, t2);
    }
    const double s = (sld - solvent)*(PI*radius*radius*length);
    F1 = 1.0e-2*s*(t1*PI_4);
    F2 = 1.0e-4*s*s*(t2*PI_4);
}

// ---- ellipsoid --------------------------------------------------------------
// Radius of the ellipse section at u = cos(angle): Re sqrt(1 + u^2 (v^2-1)),
// v = Rp/Re; the phase q*r is formed as sqrt(A + B u^2) in FP64.
__device__ __forceinline__ double ellipsoid_iqac(double qab, double qc, double sld,
                                                 double solvent, double rp, double re)
{
    const double x = sqrt_d_fast((re*qab)*(re*qab) + (rp*qc)*(rp*qc));
    const double f = (double)sph_j1c_f(x);
    const double s = (sld - solvent)*(FOUR_PI_3*rp*re*re);
    return 1.0e-4*(f*s)*(f*s);
}

__device__ __forceinline__ void ellipsoid_fq(double q, double sld, double solvent,
                                             double rp, double re, double &F1, double &F2)
{
    const double ratio = rp/re;
    const double v2m1 = ratio*ratio - 1.0;
    const Rule r = rule_for(q*fmax(rp, re));
    const double A = (q*re)*(q*re);
    const double B = A*v2m1;
    double t1 = 0.0, t2 = 0.0;
    for (int i = 0; i < r.n; ++i) {
        const double u = fma(r.z[i], 0.5, 0.5);
        const double f = (double)sph_j1c_f(sqrt_d_fast(fma(B, u*u, A)));
        const double wf = r.w[i]*f;
        t1 += wf;
        t2 = fma(wf, f, t2);
    }
    const double s = (sld - solvent)*(FOUR_PI_3*rp*re*re);
    F1 = 1.0e-2*s*(0.5*t1);
    F2 = 1.0e-4*s*s*(0.5*t2);
}

// ---- core_shell_cylinder ----------------------------------------------------
struct CoreShellCyl {
    double core_r, core_h, shell_r, shell_h;
    float core_vd, shell_vd;
    double rmax;
};

__device__ __forceinline__ CoreShellCyl core_shell_cylinder_setup(
    double core_sld, double shell_sld, double solvent_sld,
    double radius, double thickness, double length)
{
    CoreShellCyl c;
    c.core_r = radius;
    c.core_h = 0.5*length;
    c.shell_r = radius + thickness;
    c.shell_h = 0.5*length + thickness;
    c.core_vd = (float)(PI*radius*radius*length*(core_sld - shell_sld));
    c.shell_vd = (float)(PI*c.shell_r*c.shell_r*(length + 2.0*thickness)
                         *(shell_sld - solvent_sld));
    c.rmax = fmax(c.shell_r, c.shell_h);
    return c;
}

__device__ __forceinline__ float core_shell_cylinder_amp(const CoreShellCyl &c,
                                                        double qab, double qc)
{
    return c.core_vd*sinc_f(c.core_h*qc)*j1c_f(c.core_r*qab)
         + c.shell_vd*sinc_f(c.shell_h*qc)*j1c_f(c.shell_r*qab);
}

__device__ __forceinline__ double core_shell_cylinder_iqac(
    double qab, double qc, double core_sld, double shell_sld, double solvent_sld,
    double radius, double thickness, double length)
{
    const CoreShellCyl c = core_shell_cylinder_setup(core_sld, shell_sld, solvent_sld,
                                                     radius, thickness, length);
    const double f = (double)core_shell_cylinder_amp(c, qab, qc);
    return 1.0e-4*f*f;
}

__device__ __forceinline__ void core_shell_cylinder_fq(
    double q, double core_sld, double shell_sld, double solvent_sld,
    double radius, double thickness, double length, double &F1, double &F2)
{
    const CoreShellCyl c = core_shell_cylinder_setup(core_sld, shell_sld, solvent_sld,
                                                     radius, thickness, length);
    const Rule r = rule_for(q*c.rmax);
    double t1 = 0.0, t2 = 0.0;
    for (int i = 0; i < r.n; ++i) {
        const double st = r.st[i], ct = r.ct[i];
        const float f = core_shell_cylinder_amp(c, q*st, q*ct);
        const double wf = r.w[i]*st*(double)f;
        t1 += wf;
        t2 = fma(wf, (double)f, t2);
    }
    F1 = 1.0e-2*(t1*PI_4);
    F2 = 1.0e-4*(t2*PI_4);
}

}  // namespace f32c
