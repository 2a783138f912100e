"""
Seeded synthetic workloads with the shapes of the headline configurations.

No public dataset is involved: each configuration is a q grid plus a
parameter set (or a population of them) drawn with ``numpy.random`` from a
fixed seed.  ``scale`` shrinks a configuration for parity tests (fewer q
points; the dispersity mesh is kept whole unless *mesh_scale* is given).
"""

import numpy as np


def sphere_1d(nq=1000):
    """sphere 1D FP64: R=50 A gaussian pd 0.1 (35 pts, 3 sigma), 1000 log q."""
    q = np.logspace(-3, np.log10(0.5), nq)
    pars = dict(radius=50., radius_pd=0.1, radius_pd_n=35, radius_pd_nsigma=3,
                radius_pd_type='gaussian', sld=4., sld_solvent=1.,
                scale=1., background=0.001)
    return "sphere", [q], pars


def cylinder_2d(n=256, radius_n=35, length_n=35, theta_n=20, phi_n=20):
    """cylinder 2D oriented FP64: 256x256 grid over +/-0.3 1/A,
    R=20 (pd 0.1, 35), L=400 (pd 0.1, 35), theta=phi=60 with jitter
    10/15 degrees (20 pts each): 65536 q x 490000 mesh points."""
    x = np.linspace(-0.3, 0.3, n)
    qx, qy = [a.ravel() for a in np.meshgrid(x, x)]
    pars = dict(radius=20., radius_pd=0.1, radius_pd_n=radius_n,
                length=400., length_pd=0.1, length_pd_n=length_n,
                theta=60., phi=60., theta_pd=10., theta_pd_n=theta_n,
                phi_pd=15., phi_pd_n=phi_n, sld=4., sld_solvent=1.,
                scale=1., background=0.001)
    return "cylinder", [qx, qy], pars


def cylinder_2d_subgrid(n_sub, n=256, where="centre"):
    """An n_sub x n_sub block of the cylinder 2D grid (full mesh), from the
    centre of the 256x256 grid (|q| <= 0.013 1/A for 8x8: every evaluation
    takes the small-argument J1 branch) or from its corner (|q| up to
    0.42 1/A, where qab*R passes 5 and the asymptotic J1 branch runs)."""
    name, (qx, qy), pars = cylinder_2d(n)
    qx = qx.reshape(n, n)
    qy = qy.reshape(n, n)
    lo = (n - n_sub)//2 if where == "centre" else 0
    return name, [qx[lo:lo+n_sub, lo:lo+n_sub].ravel(),
                  qy[lo:lo+n_sub, lo:lo+n_sub].ravel()], pars


def cylinder_2d_strided(stride, n=256):
    """Every stride-th row and column of the cylinder 2D grid (full mesh):
    a sample with the branch mix of the whole grid (16 -> 16x16 points)."""
    name, (qx, qy), pars = cylinder_2d(n)
    qx = qx.reshape(n, n)[::stride, ::stride].ravel()
    qy = qy.reshape(n, n)[::stride, ::stride].ravel()
    return name, [qx, qy], pars


def cylinder_j1_large_fraction(qx, qy, pars):
    """Fraction of the (q, mesh point) evaluations of the cylinder 2D
    workload whose J1 argument qab*R exceeds 5, i.e. that take the
    asymptotic branch of the reference's J1 (models/lib/sas_J1.c).  Computed
    on the host from the same mesh: orientation jitter (theta, phi) and
    radius only; length does not enter qab."""
    from .direct_model import get_mesh
    from .core import load_model_info
    info = load_model_info("cylinder")
    mesh = {p.name: m for p, m in zip(info.parameters.call_parameters,
                                      get_mesh(info, pars, dim='2d'))}
    radius = np.asarray(mesh["radius"][1])
    dtheta = np.asarray(mesh["theta"][1])
    dphi = np.asarray(mesh["phi"][1])
    th, ph = np.radians(pars["theta"]), np.radians(pars["phi"])
    dt, dp = np.meshgrid(np.radians(dtheta), np.radians(dphi), indexing="ij")
    dt, dp = dt.ravel(), dp.ravel()
    # third row of the jitter x view rotation (kernel_iq.c qac_rotation)
    V31, V32 = np.sin(th)*np.cos(ph), np.sin(ph)*np.sin(th)
    V11, V12 = np.cos(ph)*np.cos(th), np.sin(ph)*np.cos(th)
    V21, V22 = -np.sin(ph), np.cos(ph)
    J31, J32, J33 = np.sin(dt), -np.sin(dp)*np.cos(dt), np.cos(dp)*np.cos(dt)
    R31 = J31*V11 + J32*V21 + J33*V31
    R32 = J31*V12 + J32*V22 + J33*V32
    qc = np.outer(qx, R31) + np.outer(qy, R32)
    qab = np.sqrt(np.maximum((qx**2 + qy**2)[:, None] - qc**2, 0.0))
    big = (qab[:, :, None]*radius[None, None, :] > 5.0)
    return float(big.mean())


def core_shell_sphere_magnetic(n=128, seed=0, radius_n=51, thickness_n=21):
    """core_shell_sphere 2D magnetic: 128x128 grid over +/-0.1 1/A,
    R=60 (lognormal pd 0.2, 51 pts, 3 sigma), t=10 (gaussian pd 0.1, 21),
    slds 1/2/3 with M0 ~ U[0,3], mtheta ~ U[0,180], mphi ~ U[0,360];
    up_frac_i=0.9, up_frac_f=0.8 and up_angle=45 (= up_theta 90,
    up_phi 45 in the current parameter names)."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-0.1, 0.1, n)
    qx, qy = [a.ravel() for a in np.meshgrid(x, x)]
    pars = dict(radius=60., radius_pd=0.2, radius_pd_n=radius_n,
                radius_pd_nsigma=3, radius_pd_type='lognormal',
                thickness=10., thickness_pd=0.1, thickness_pd_n=thickness_n,
                thickness_pd_type='gaussian',
                sld_core=1., sld_shell=2., sld_solvent=3.,
                up_frac_i=0.9, up_frac_f=0.8, up_theta=90., up_phi=45.,
                scale=1., background=0.001)
    for sld in ("sld_core", "sld_shell", "sld_solvent"):
        pars[sld + "_M0"] = float(rng.uniform(0, 3))
        pars[sld + "_mtheta"] = float(rng.uniform(0, 180))
        pars[sld + "_mphi"] = float(rng.uniform(0, 360))
    return "core_shell_sphere", [qx, qy], pars


# ------------------------------------------------------ fit population ----

POP_MODELS = ("ellipsoid", "core_shell_cylinder")
POP_SIZE_PARS = {
    "ellipsoid": ("radius_polar", "radius_equatorial"),
    "core_shell_cylinder": ("radius", "thickness", "length"),
}


def _log_uniform(rng, lo, hi):
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def population(n_sets=4096, seed=1, nq_range=(100, 2000), max_pd_n=71,
               pd_width=(0.05, 0.3)):
    """
    A bumps/DREAM-like population: half ellipsoid, half core_shell_cylinder
    (1D), each set with its own q vector (length U{100..2000}, log spaced
    1e-3..0.6), radii log-U[10,500], lengths log-U[20,2000], slds U[-1,7],
    and 1..(2 or 3) polydisperse size parameters with gaussian pd of width
    U[0.05,0.3] and U{1..71} points.

    Returns a list of (model, q, pars).
    """
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_sets):
        model = POP_MODELS[k % 2]
        nq = int(rng.integers(nq_range[0], nq_range[1] + 1))
        q = np.logspace(-3, np.log10(0.6), nq)
        if model == "ellipsoid":
            pars = dict(radius_polar=_log_uniform(rng, 10, 500),
                        radius_equatorial=_log_uniform(rng, 10, 500),
                        sld=float(rng.uniform(-1, 7)),
                        sld_solvent=float(rng.uniform(-1, 7)))
        else:
            pars = dict(radius=_log_uniform(rng, 10, 500),
                        thickness=_log_uniform(rng, 10, 500),
                        length=_log_uniform(rng, 20, 2000),
                        sld_core=float(rng.uniform(-1, 7)),
                        sld_shell=float(rng.uniform(-1, 7)),
                        sld_solvent=float(rng.uniform(-1, 7)))
        size_pars = POP_SIZE_PARS[model]
        n_active = int(rng.integers(1, len(size_pars) + 1))
        chosen = rng.choice(len(size_pars), size=n_active, replace=False)
        for c in sorted(chosen):
            p = size_pars[c]
            pars[p + "_pd"] = float(rng.uniform(*pd_width))
            pars[p + "_pd_n"] = int(rng.integers(1, max_pd_n + 1))
            pars[p + "_pd_type"] = "gaussian"
        pars["scale"] = 1.0
        pars["background"] = 0.0
        out.append((model, q, pars))
    return out
