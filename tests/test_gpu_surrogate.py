"""
The learned surrogate end to end on a reduced budget: data from the plain
kernels, training with the tensor-core kernels, calibration on held-out sets
judged by the plain FP64 kernel, and what the network gains over the plain
method: throughput at a fixed accuracy, with the automatic fallback keeping
the accepted points within tolerance.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_gain(cuda):
    from sasmodels_b200.surrogate import train_and_evaluate
    # a net trained for seconds is far from the full one: the gate is
    # calibrated here for 1 % violations among the accepted points (the
    # full configuration uses 0.05 %)
    S, rep = train_and_evaluate(n_train_sets=3000, nq=400, epochs=4, n_holdout_sets=600,
                                seed=0, low_pd_frac=0.4, alpha=0.01)
    assert S.net.errors() == 0
    # a few seconds of training already predicts log I to a few percent
    assert rep["net_median_err"] < 0.05, rep
    # the network alone is far faster than the plain kernel on the same points
    assert rep["net_only_speedup"] > 10, rep
    # with the error gate, the returned curve is within 5 % (log I) almost
    # everywhere: mistrusted points come from the plain kernel
    op = rep["operating_points"]["0.05"]
    assert op["frac_within"] > 0.99, rep
    assert 0.0 <= op["fallback_frac"] < 1.0
    # the calibrated gate keeps the accepted points within tolerance (the
    # bound is statistical: 400 calibration sets at this size)
    assert op["accepted_frac_within"] > 0.98, rep


def test_surrogate_fallback_is_exact_where_used(cuda):
    """Points outside the training domain always fall back and come back as
    the plain kernel's values."""
    from sasmodels_b200.surrogate import Surrogate, flatten, plain_unit_iq, sample_q, sample_sets
    S = Surrogate(seed=3)
    rng = np.random.default_rng(4)
    sets = sample_sets(4, rng)
    sets["radius"][:] = 400.0              # outside the [10, 300] training range
    qs = [sample_q(50, rng) for _ in range(4)]
    cols = flatten(sets, qs)
    from sasmodels_b200.surrogate import MLP
    S.gate = MLP(seed=5, stream=S.net.stream)
    S.cal_tols = np.array([1e-3, 1.0])     # trust everything inside the domain
    S.cal_thresh = np.array([np.inf, np.inf])
    I, back = S.iq(cols, tol=0.01)
    assert back.all()
    ref = np.concatenate(plain_unit_iq(sets, qs, form="float32c"))*np.repeat(
        sets["contrast"]**2, 50)
    np.testing.assert_allclose(I, ref, rtol=1e-12)
