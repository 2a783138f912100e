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

// ---- quadrature functors ---------------------------------------------------
// A 1D orientation/shape average is split into
//   setup(q, v)            per (q, mesh point) constants and the Gauss rule,
//   nodes(S)               number of rule points,
//   node(S, i, t1, t2)     add point i's w*F and w*F^2 to FP64 sums,
//   finish(S, t1, t2, ..)  scale to <F>, <F^2>,
// so the same arithmetic serves one lane walking all points (quad_fq) and a
// warp sharing the points of one (q, mesh point) in the batched kernel.

template <class Q>
__device__ __forceinline__ void quad_fq(double q, const double *v, double &F1, double &F2)
{
    const typename Q::S s = Q::setup(q, v);
    double t1 = 0.0, t2 = 0.0;
    const int n = Q::nodes(s);
    for (int i = 0; i < n; ++i) Q::node(s, i, t1, t2);
    Q::finish(s, t1, t2, F1, F2);
}

// sphere (sphere.c:13-20): v = sld, sld_solvent, radius; one "node"
struct QuadSphere {
    struct S { double q, r, s; };
    __device__ static S setup(double q, const double *v)
    {
        return S{q, v[2], (v[0] - v[1])*(FOUR_PI_3*v[2]*v[2]*v[2])};
    }
    __device__ static int nodes(const S &) { return 1; }
    __device__ static void node(const S &s, int, double &t1, double &t2)
    {
        const double f = s.s*(double)sph_j1c_f(s.q*s.r);
        t1 += f;
        t2 = fma(f, f, t2);
    }
    __device__ static void finish(const S &, double t1, double t2, double &F1, double &F2)
    {
        F1 = 1.0e-2*t1;
        F2 = 1.0e-4*t2;
    }
};

// core_shell_sphere (core_shell_sphere.c:19-30, lib/core_shell.c:8-30):
// v = radius, thickness, sld_core, sld_shell, sld_solvent; one "node"
struct QuadCoreShellSphere {
    struct S { double q, r, rt; float core, shell; };
    __device__ static S setup(double q, const double *v)
    {
        const double rt = v[0] + v[1];
        return S{q, v[0], rt, (float)(FOUR_PI_3*v[0]*v[0]*v[0]*(v[2] - v[3])),
                 (float)(FOUR_PI_3*rt*rt*rt*(v[3] - v[4]))};
    }
    __device__ static int nodes(const S &) { return 1; }
    __device__ static void node(const S &s, int, double &t1, double &t2)
    {
        const double f = (double)(s.core*sph_j1c_f(s.q*s.r) + s.shell*sph_j1c_f(s.q*s.rt));
        t1 += f;
        t2 = fma(f, f, t2);
    }
    __device__ static void finish(const S &, double t1, double t2, double &F1, double &F2)
    {
        F1 = 1.0e-2*t1;
        F2 = 1.0e-4*t2;
    }
};

// The magnetic form of core_shell_sphere with its spin channels sharing one
// evaluation of the two Bessel terms (QuadCoreShellSphere's arithmetic, the
// channel's effective slds in place of v[2..4]): sum over the channels c
// with chan_w[c] > 0 of chan_w[c] * F^2.  mag_par(k) gives the slot of
// magnetic sld k in v.
template <class MagPar>
__device__ __forceinline__ double core_shell_sphere_channels(double q, const double *v,
                                                             const double (*eff)[3],
                                                             const double *chan_w, MagPar mag_par)
{
    const double rt = v[0] + v[1];
    const float bc = sph_j1c_f(q*v[0]);
    const float bs = sph_j1c_f(q*rt);
    const double vc = FOUR_PI_3*v[0]*v[0]*v[0];
    const double vs = FOUR_PI_3*rt*rt*rt;
    double F2 = 0.0;
    #pragma unroll
    for (int c = 0; c < 5; ++c) {
        if (chan_w[c] > 0.0) {
            double sl[5] = {v[0], v[1], v[2], v[3], v[4]};
            #pragma unroll
            for (int k = 0; k < 3; ++k) sl[mag_par(k)] = eff[c][k];
            const float core = (float)(vc*(sl[2] - sl[3]));
            const float shell = (float)(vs*(sl[3] - sl[4]));
            const double f = (double)(core*bc + shell*bs);
            F2 += chan_w[c]*(1.0e-4*fma(f, f, 0.0));
        }
    }
    return F2;
}

// cylinder (cylinder.c:55-88): v = sld, sld_solvent, radius, length, ...
struct QuadCylinder {
    struct S { double qr, qh, s; Rule r; };
    __device__ static S setup(double q, const double *v)
    {
        const double radius = v[2], length = v[3];
        return S{q*radius, q*0.5*length, (v[0] - v[1])*(PI*radius*radius*length),
                 rule_for(q*fmax(radius, 0.5*length))};
    }
    __device__ static int nodes(const S &s) { return s.r.n; }
    __device__ static void node(const S &s, int i, double &t1, double &t2)
    {
        const double st = s.r.st[i], ct = s.r.ct[i];
        const float form = j1c_f(s.qr*st)*sinc_f(s.qh*ct);
        const double wf = s.r.w[i]*st*(double)form;
        t1 += wf;
        t2 = fma(wf, (double)form, t2);
    }
    __device__ static void finish(const S &s, double t1, double t2, double &F1, double &F2)
    {
        F1 = 1.0e-2*s.s*(t1*PI_4);
        F2 = 1.0e-4*s.s*s.s*(t2*PI_4);
    }
};

__device__ __forceinline__ double cylinder_iqac(double qab, double qc, double sld,
                                                double solvent, double radius, double length)
{
    const float form = j1c_f(qab*radius)*sinc_f(qc*0.5*length);
    const double s = (sld - solvent)*(PI*radius*radius*length);
    const double a = s*(double)form;
    return 1.0e-4*a*a;
}

// ellipsoid (ellipsoid.c:50-91): v = sld, sld_solvent, radius_polar,
// radius_equatorial, ...  The section radius Re sqrt(1 + u^2 (v^2-1)) at
// u = cos(angle) enters as the phase q r = sqrt(A + B u^2), formed in FP64.
struct QuadEllipsoid {
    struct S { double A, B, s; Rule r; };
    __device__ static S setup(double q, const double *v)
    {
        const double rp = v[2], re = v[3];
        const double ratio = rp/re;
        const double A = (q*re)*(q*re);
        return S{A, A*(ratio*ratio - 1.0), (v[0] - v[1])*(FOUR_PI_3*rp*re*re),
                 rule_for(q*fmax(rp, re))};
    }
    __device__ static int nodes(const S &s) { return s.r.n; }
    __device__ static void node(const S &s, int i, double &t1, double &t2)
    {
        const double u = fma(s.r.z[i], 0.5, 0.5);
        const double f = (double)sph_j1c_f(sqrt_d_fast(fma(s.B, u*u, s.A)));
        const double wf = s.r.w[i]*f;
        t1 += wf;
        t2 = fma(wf, f, t2);
    }
    __device__ static void finish(const S &s, double t1, double t2, double &F1, double &F2)
    {
        F1 = 1.0e-2*s.s*(0.5*t1);
        F2 = 1.0e-4*s.s*s.s*(0.5*t2);
    }
};

__device__ __forceinline__ double ellipsoid_iqac(double qab, double qc, double sld,
                                                 double solvent, double rp, double re)
{
    const double x = sqrt_d_fast((re*qab)*(re*qab) + (rp*qc)*(rp*qc));
    const double f = (double)sph_j1c_f(x);
    const double s = (sld - solvent)*(FOUR_PI_3*rp*re*re);
    return 1.0e-4*(f*s)*(f*s);
}

// core_shell_cylinder (core_shell_cylinder.c:4-7, 60-123): v = sld_core,
// sld_shell, sld_solvent, radius, thickness, length, ...
struct CoreShellCyl {
    double core_r, core_h, shell_r, shell_h;
    float core_vd, shell_vd;
    double rmax;
};

__device__ __forceinline__ CoreShellCyl core_shell_cylinder_setup(const double *v)
{
    const double radius = v[3], thickness = v[4], length = v[5];
    CoreShellCyl c;
    c.core_r = radius;
    c.core_h = 0.5*length;
    c.shell_r = radius + thickness;
    c.shell_h = 0.5*length + thickness;
    c.core_vd = (float)(PI*radius*radius*length*(v[0] - v[1]));
    c.shell_vd = (float)(PI*c.shell_r*c.shell_r*(length + 2.0*thickness)*(v[1] - v[2]));
    c.rmax = fmax(c.shell_r, c.shell_h);
    return c;
}

__device__ __forceinline__ float core_shell_cylinder_amp(const CoreShellCyl &c,
                                                        double qab, double qc)
{
    return c.core_vd*sinc_f(c.core_h*qc)*j1c_f(c.core_r*qab)
         + c.shell_vd*sinc_f(c.shell_h*qc)*j1c_f(c.shell_r*qab);
}

struct QuadCoreShellCylinder {
    struct S { double q; CoreShellCyl c; Rule r; };
    __device__ static S setup(double q, const double *v)
    {
        const CoreShellCyl c = core_shell_cylinder_setup(v);
        return S{q, c, rule_for(q*c.rmax)};
    }
    __device__ static int nodes(const S &s) { return s.r.n; }
    __device__ static void node(const S &s, int i, double &t1, double &t2)
    {
        const double st = s.r.st[i], ct = s.r.ct[i];
        const float f = core_shell_cylinder_amp(s.c, s.q*st, s.q*ct);
        const double wf = s.r.w[i]*st*(double)f;
        t1 += wf;
        t2 = fma(wf, (double)f, t2);
    }
    __device__ static void finish(const S &, double t1, double t2, double &F1, double &F2)
    {
        F1 = 1.0e-2*(t1*PI_4);
        F2 = 1.0e-4*(t2*PI_4);
    }
};

__device__ __forceinline__ double core_shell_cylinder_iqac(double qab, double qc, const double *v)
{
    const double f = (double)core_shell_cylinder_amp(core_shell_cylinder_setup(v), qab, qc);
    return 1.0e-4*f*f;
}

}  // namespace f32c
