"""
CPU tests pinning the restated oracle (oracle/sas_oracle.c) to the reference:
it must reproduce the reference DLL's raw result vectors bitwise, at any
thread count, including restarts and cutoffs.
"""

import numpy as np
import pytest

from helpers import (MODELS, golden, interleave, load_info, marshal, nout_of,
                     variant)
from sasmodels_b200 import workloads


def _port(name):
    from oracle import port
    return port.load(name)


@pytest.mark.parametrize("name", MODELS)
@pytest.mark.parametrize("threads", [1, 4])
def test_port_matches_recorded_dll(name, threads):
    info = load_info(name)
    for case in golden(name)["dll"]:
        nout = nout_of(info, case["dim"])
        raw = _port(name).call(variant(case["dim"], case["magnetic"]),
                               interleave(case["q"]), case["details"],
                               np.array(case["values"]), nout, threads=threads)
        np.testing.assert_array_equal(raw, np.array(case["raw"]))


def _both(name, qv, pars, cutoff=0.0, reff_mode=0, threads=3):
    from oracle import refdll
    info = load_info(name)
    details, values, magnetic = marshal(info, pars, qv)
    dim = '2d' if len(qv) == 2 else '1d'
    var, nout = variant(dim, magnetic), nout_of(info, dim)
    q = interleave(qv)
    a = _port(name).call(var, q, details.buffer, values, nout, cutoff, reff_mode, threads)
    b = refdll.load(name).call(var, q, details.buffer, values, nout, cutoff, reff_mode)
    return a, b


@pytest.mark.parametrize("k", range(6))
def test_port_matches_live_dll_population(k):
    name, q, pars = workloads.population(n_sets=6, seed=1, max_pd_n=6)[k]
    a, b = _both(name, [q[::7]], pars)
    np.testing.assert_array_equal(a, b)


def test_port_matches_live_dll_cutoff_reff():
    q = np.logspace(-3, -0.5, 40)
    pars = dict(radius=30., radius_pd=0.2, radius_pd_n=25, length=200.,
                length_pd=0.3, length_pd_n=25)
    for cutoff, mode in ((1e-4, 1), (0.0, 7), (3e-3, 2)):
        a, b = _both("cylinder", [q], pars, cutoff, mode)
        np.testing.assert_array_equal(a, b)


def test_port_matches_live_dll_magnetic_and_oriented():
    _, qv, pars = workloads.core_shell_sphere_magnetic(n=7, radius_n=9, thickness_n=5)
    a, b = _both("core_shell_sphere", qv, pars)
    np.testing.assert_array_equal(a, b)
    _, qv, pars = workloads.cylinder_2d(n=7, radius_n=5, length_n=5, theta_n=4, phi_n=3)
    a, b = _both("cylinder", qv, pars)
    np.testing.assert_array_equal(a, b)


def test_port_restart():
    """pd_start > 0 continues the sums in the result vector."""
    from oracle import refdll
    name, qv, pars = workloads.cylinder_2d(n=5, radius_n=5, length_n=4, theta_n=3, phi_n=3)
    info = load_info(name)
    details, values, magnetic = marshal(info, pars, qv)
    q = interleave(qv)
    n = details.num_eval
    port = _port(name)
    part = port.call("Iqxy", q, details.buffer, values, 1, pd_start=0, pd_stop=n//2)
    part = port.call("Iqxy", q, details.buffer, values, 1, pd_start=n//2, pd_stop=n,
                     result=part)
    ref = refdll.load(name).call("Iqxy", q, details.buffer, values, 1)
    np.testing.assert_array_equal(part, ref)
