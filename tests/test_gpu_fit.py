"""
The fit step of a whole population on the device: batched theory ->
pinhole smearing -> nllf (bumps_model.py:263-282), against the same chain
on the host from the reference DLL (oracle) and the dense resolution matrix.
"""

import numpy as np
import pytest

from helpers import load_info, marshal, normalise, reference_raw

pytestmark = pytest.mark.gpu


def _population(q_calc, n=12, seed=4):
    rng = np.random.default_rng(seed)
    sets = []
    for k in range(n):
        sets.append((q_calc, dict(radius_polar=float(rng.uniform(20, 80)),
                                  radius_equatorial=float(rng.uniform(20, 80)),
                                  radius_polar_pd=0.1, radius_polar_pd_n=11,
                                  sld=4.0, sld_solvent=1.0, scale=float(rng.uniform(0.5, 2)),
                                  background=0.01)))
    return sets


@pytest.mark.parametrize("smear", [False, True])
def test_population_nllf(cuda, smear):
    from oracle import resolution_ref
    from sasmodels_b200.batch import Population
    from sasmodels_b200.resolution import Pinhole1D
    q = np.logspace(-2.5, np.log10(0.4), 90)
    res = Pinhole1D(q, 0.06*q) if smear else None
    q_calc = res.q_calc if smear else q
    sets = _population(q_calc)
    info = load_info("ellipsoid")
    # data: one member's curve with noise, 5 % errors
    rng = np.random.default_rng(9)
    truth = dict(sets[3][1], radius_polar=55.0)
    raw = reference_raw("ellipsoid", info, [q_calc], truth)
    _, v, _ = marshal(info, truth, [q_calc])
    I_true = normalise(raw, 2, len(q_calc), v)["I"]
    W = resolution_ref.pinhole_matrix(res._signed_q_calc, q, 0.06*q) if smear else None
    if smear:
        I_true = resolution_ref.smear_1d(W, I_true)
    dI = 0.05*I_true
    Iq = I_true + dI*rng.normal(size=I_true.size)
    pop = Population("ellipsoid", sets, form="double")
    pop.run()
    got = pop.nllf(Iq, dI, resolution=res)
    for (qs, pars), g in zip(sets, got):
        raw = reference_raw("ellipsoid", info, [qs], pars)
        _, v, _ = marshal(info, pars, [qs])
        th = normalise(raw, 2, len(qs), v)["I"]
        if smear:
            th = resolution_ref.smear_1d(W, th)
        want = 0.5*np.sum(((th - Iq)/dI)**2)
        assert abs(g - want) <= 1e-10*want, (g, want)
