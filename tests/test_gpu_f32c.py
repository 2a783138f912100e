"""
GPU accuracy of the FP32-compensated form against the FP64 reference DLL.

Bar: max relative error of every F^2 / I(q) slot <= 1e-5 (and <F> within
1e-5 of its Cauchy-Schwarz scale), the ceiling the FP32c form is built to.
"""

import numpy as np
import pytest

from helpers import (MODELS, compare_raw, golden, load_info, marshal, nout_of,
                     reference_raw)
from sasmodels_b200 import load_model, workloads

pytestmark = pytest.mark.gpu

RTOL_F32C = 1e-5


def f32c_raw(name, q_vectors, pars, cutoff=0.0, reff_mode=0):
    model = load_model(name, dtype="float32c")
    assert model.form == "float32c"
    kernel = model.make_kernel([np.asarray(v, 'd') for v in q_vectors])
    details, values, magnetic = marshal(model.info, pars, q_vectors)
    kernel._call_kernel(details, values, cutoff, magnetic, reff_mode)
    nout = nout_of(model.info, kernel.dim)
    nq = kernel.q_input.nq
    return np.concatenate([kernel.result[:nout*nq], kernel.result[nout*nq:nout*nq+4]]), nout, nq


def assert_f32c(name, q_vectors, pars, threads=8, rtol=RTOL_F32C):
    info = load_info(name)
    ours, nout, nq = f32c_raw(name, q_vectors, pars)
    ref = reference_raw(name, info, q_vectors, pars, threads=threads)
    worst, f2rel = compare_raw(ours, ref, nout, nq, rtol)
    assert worst <= 1.0, "%s: %.3g x tol (max F^2 rel %.3g)" % (name, worst, f2rel)
    return f2rel


@pytest.mark.parametrize("name", MODELS)
def test_f32c_golden_cases(cuda, name):
    for case in golden(name)["dll"]:
        info = load_info(name)
        ours, nout, nq = f32c_raw(name, case["q"], case["pars"])
        worst, f2rel = compare_raw(ours, np.array(case["raw"]), nout, nq, RTOL_F32C)
        assert worst <= 1.0, (name, case["dim"], worst, f2rel)


@pytest.mark.parametrize("k", range(12))
def test_f32c_population_members(cuda, k):
    """Fit-population members (ellipsoid / core_shell_cylinder 1D, adaptive
    quadrature up to 5000 points), reduced mesh."""
    name, q, pars = workloads.population(n_sets=12, seed=1, max_pd_n=7)[k]
    assert_f32c(name, [q], pars)


def test_f32c_large_qr(cuda):
    """Phases of several hundred radians (5000-point rule)."""
    q = np.logspace(-2, np.log10(0.6), 60)
    assert_f32c("core_shell_cylinder", [q],
                dict(radius=300., thickness=200., length=1900., sld_core=6.,
                     sld_shell=-0.5, sld_solvent=2., radius_pd=0.1, radius_pd_n=3))
    assert_f32c("ellipsoid", [q], dict(radius_polar=480., radius_equatorial=30.,
                                       radius_polar_pd=0.1, radius_polar_pd_n=5))


def test_f32c_magnetic_config(cuda):
    """core_shell_sphere 2D magnetic (full 1071-point mesh, q subsample)."""
    name, (qx, qy), pars = workloads.core_shell_sphere_magnetic(n=128)
    sub = np.arange(0, 128*128, 97)
    assert_f32c(name, [qx[sub], qy[sub]], pars)


def test_f32c_cylinder_2d(cuda):
    name, qv, pars = workloads.cylinder_2d_subgrid(6)
    assert_f32c(name, qv, pars)


def test_f32c_sphere_config(cuda):
    name, qv, pars = workloads.sphere_1d()
    assert_f32c(name, qv, pars)
