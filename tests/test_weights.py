"""
Dispersity meshes (sasmodels_b200.weights) against the reference's
``sasmodels.weights.get_weights``: bit for bit on the recorded fixtures
(tests/golden/weights.json, made by tests/golden/make_weights_golden.py from
the reference package), and on randomised cases against the live reference
where it is importable.
"""

import json
import os
import sys

import numpy as np
import pytest

from sasmodels_b200 import weights
from sasmodels_b200.build import locate_sasmodels

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "weights.json")


def _cases():
    with open(GOLDEN) as fid:
        return json.load(fid)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: "%s-%s-%s-%s" % (
    c["kind"], c["npts"], c["width"], c["value"]))
def test_weights_match_recorded_reference(case):
    limits = tuple(float(v) for v in case["limits"])
    args = (case["kind"], case["npts"], case["width"], case["nsigmas"], case["value"],
            limits, case["relative"])
    if "error" in case:
        with pytest.raises(ZeroDivisionError):
            weights.get_weights(*args)
        return
    with np.errstate(all="ignore"):
        x, w = weights.get_weights(*args)
    np.testing.assert_array_equal(x, np.array(case["x"]))
    np.testing.assert_array_equal(w, np.array(case["w"]))


def test_defaults_and_errors():
    # default npts and nsigmas of each distribution, as the reference's
    x, _ = weights.dispersion("lognormal", None, 0.1, None, 50.0, (0, np.inf), True)
    assert len(x) == 80 and x.min() == pytest.approx(50.0*(1 - 0.8))
    x, _ = weights.dispersion("rectangle", None, 0.1, None, 50.0, (0, np.inf), True)
    assert len(x) == 35
    with pytest.raises(ValueError, match="array"):
        weights.get_weights("array", 3, 0.1, 3, 1.0, (0, 1), True)
    with pytest.raises(ValueError, match="unknown"):
        weights.get_weights("cauchy", 3, 0.1, 3, 1.0, (0, 1), True)


@pytest.mark.skipif(locate_sasmodels() is None, reason="sasmodels not importable")
def test_weights_match_live_reference():
    path = locate_sasmodels()
    if path not in sys.path:
        sys.path.insert(0, path)
    from sasmodels import weights as ref
    rng = np.random.default_rng(7)
    for _ in range(300):
        kind = rng.choice(list(weights.SPECS))
        npts = int(rng.integers(1, 90))
        width = float(rng.choice([0.0, rng.uniform(0.01, 0.6)]))
        nsigmas = float(rng.uniform(1, 8))
        value = float(rng.uniform(1, 500))
        lb = float(rng.choice([0.0, -np.inf, value*rng.uniform(0.5, 1)]))
        ub = float(rng.choice([np.inf, value*rng.uniform(1, 1.5)]))
        args = (kind, npts, width, nsigmas, value, (lb, ub), True)
        with np.errstate(all="ignore"):
            x0, w0 = ref.get_weights(*args)
            x1, w1 = weights.get_weights(*args)
        np.testing.assert_array_equal(x1, x0)
        np.testing.assert_array_equal(w1, w0)
