"""
Generate tests/golden/weights.json from the reference package: the points
and normalised weights of ``sasmodels.weights.get_weights`` for every
distribution the plugin API offers, over cases that exercise the default
widths, truncation at parameter limits, absolute (orientation) jitter, the
positive-domain clipping of lognormal and schulz, and the degenerate
zero-width and one-point meshes.

    PYTHONPATH=<sasmodels source tree> python tests/golden/make_weights_golden.py

The tests read only the JSON output.
"""

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INF = float("inf")

#: (npts, width, nsigmas, value, (lb, ub), relative)
CASES = [
    (35, 0.1, 3, 50.0, (0, INF), True),
    (35, 0.5, 3, 1.0, (0, INF), True),          # truncated at the lower limit
    (71, 0.3, 3, 400.0, (0, INF), True),
    (20, 10.0, 3, 60.0, (-180, 180), False),    # orientation jitter
    (21, 45.0, 3, 10.0, (-90, 90), False),      # jitter clipped at +/- 90
    (51, 0.2, 8, 60.0, (0, INF), True),
    (80, 0.05, None, 120.0, (0, INF), True),    # default nsigmas
    (7, 0.25, 2.5, 5.0, (4.0, 6.0), True),      # both limits inside the range
    (35, 0.0, 3, 20.0, (0, INF), True),         # zero width: the value alone
    (1, 0.2, 3, 20.0, (0, INF), True),          # one point
    (35, 0.2, 3, -1.0, (0, INF), True),         # centre outside the limits
    (35, 1.5, 3, 2.0, (-INF, INF), True),       # wide: crosses zero
]


def main():
    from sasmodels import weights
    out = []
    for kind in ("gaussian", "uniform", "rectangle", "lognormal", "schulz", "boltzmann"):
        for npts, width, nsigmas, value, limits, relative in CASES:
            if nsigmas is None:
                nsigmas = weights.MODELS[kind].default["nsigmas"]
            try:
                with np.errstate(all="ignore"):
                    x, w = weights.get_weights(kind, npts, width, nsigmas, value,
                                               limits, relative)
                rec = {"x": [float(v) for v in x], "w": [float(v) for v in w]}
            except Exception as exc:        # recorded: the same error is expected
                rec = {"error": type(exc).__name__}
            out.append({"kind": kind, "npts": npts, "width": width, "nsigmas": nsigmas,
                        "value": value, "limits": [repr(v) for v in limits],
                        "relative": relative, **rec})
    with open(os.path.join(HERE, "weights.json"), "w") as fid:
        json.dump(out, fid, indent=0)
    print("wrote %d cases" % len(out))


if __name__ == "__main__":
    main()
