"""
Dispersity meshes: a parameter's value and distribution -> (points, weights).

The kernels integrate over the points and weights given here, so they must
be the ones the reference's plugin API produces (``sasmodels/weights.py``:
distributions :86-220, defaults and truncation :21-83, normalisation
:264-291), bit for bit: each weight function below evaluates the same
expression as the reference's in the same operation order, on points from
the same ``numpy.linspace`` call.  The organisation is this module's own: a
table of distribution specs (default size and width in sigmas, node rule,
weight function, domain) over two node rules, and one function that applies
a spec.

Volume-type parameters take a width relative to their value; orientation
jitter is absolute and centred on zero.  A distribution of zero width (or
fewer than two points) is its centre alone, if the centre lies within the
parameter's limits.  Points outside the limits are dropped.
"""

from collections import namedtuple

import numpy as np
from scipy.special import gammaln

# ------------------------------------------------------------ node rules ---


def _nodes_sigma(center, sigma, npts, nsigmas):
    """npts points evenly spaced over center +/- nsigmas*sigma."""
    return center + np.linspace(-nsigmas*sigma, +nsigmas*sigma, npts)


def _nodes_width(center, sigma, npts, nsigmas):
    """npts points evenly spaced over center +/- sigma (nsigmas unused)."""
    return np.linspace(center - sigma, center + sigma, npts)


# ------------------------------------------------------ weight functions ---
# Unnormalised densities at the points x for a distribution of centre c and
# width s (the expressions of sasmodels/weights.py, operation by operation).

def _w_gaussian(x, c, s):
    return np.exp((x - c)**2 / (-2.0*s*s))


def _w_flat(x, c, s):
    return np.ones_like(x)


def _w_lognormal(x, c, s):
    sig = np.fabs(s/c)
    return np.exp(-0.5*((np.log(x) - np.log(c))/sig)**2)/(x*sig)


def _w_schulz(x, c, s):
    R = x/c
    z = (c/s)**2
    return np.exp(z*np.log(z) + (z - 1)*np.log(R) - R*z - np.log(c) - gammaln(z))


def _w_boltzmann(x, c, s):
    return np.exp(-np.abs(x - c) / np.abs(s))


#: npts, nsigmas: defaults; nodes: node rule; weight: density;
#: positive: points are taken over [max(lb, 1e-8), max(ub, 1e-8)] (the
#: densities with a log); box: also drop points farther than |s| sqrt(3)
#: from the centre (the rectangle of standard deviation s)
Spec = namedtuple("Spec", "npts nsigmas nodes weight positive box")

SPECS = {
    "gaussian": Spec(35, 3, _nodes_sigma, _w_gaussian, False, False),
    "uniform": Spec(35, None, _nodes_width, _w_flat, False, False),
    "rectangle": Spec(35, 1.73205, _nodes_sigma, _w_flat, False, True),
    "lognormal": Spec(80, 8, _nodes_sigma, _w_lognormal, True, False),
    "schulz": Spec(80, 8, _nodes_sigma, _w_schulz, True, False),
    "boltzmann": Spec(35, 3, _nodes_sigma, _w_boltzmann, False, False),
}

#: distribution names in the order the reference lists them
#: (sasmodels/weights.py:225-233); "array" (user-supplied points and
#: weights) is handled by the caller, not by get_weights
NAMES = ("rectangle", "uniform", "array", "lognormal", "gaussian", "schulz", "boltzmann")


def dispersion(kind, npts, width, nsigmas, center, limits, relative):
    """Unnormalised (points, weights) of distribution *kind* for a
    parameter at *center* with *limits* = (lb, ub).  *npts*, *width* and
    *nsigmas* may be None for the distribution's defaults (width 0)."""
    if kind == "array":
        raise ValueError("array dispersity: pass the points and weights directly")
    try:
        spec = SPECS[kind]
    except KeyError:
        raise ValueError("unknown dispersity distribution %r" % (kind,)) from None
    npts = spec.npts if npts is None else int(npts)
    width = 0 if width is None else width
    nsigmas = spec.nsigmas if nsigmas is None else nsigmas
    lb, ub = limits
    sigma = width*center if relative else width
    if not relative:
        center = 0
    if sigma == 0 or npts < 2:
        if lb <= center <= ub:
            return np.array([center], 'd'), np.array([1.], 'd')
        return np.array([], 'd'), np.array([], 'd')
    if spec.positive:
        lb, ub = max(lb, 1e-8), max(ub, 1e-8)
    x = spec.nodes(center, sigma, npts, nsigmas)
    x = x[(x >= lb) & (x <= ub)]
    if spec.box:
        x = x[np.fabs(x - center) <= np.fabs(sigma)*np.sqrt(3.0)]
    return x, spec.weight(x, center, sigma)


def get_weights(kind, npts, width, nsigmas, value, limits, relative):
    """(points, weights) of one polydisperse parameter, the weights
    normalised to sum to one (the call the reference's direct_model makes,
    sasmodels/weights.py:264-291)."""
    x, w = dispersion(kind, npts, width, nsigmas, value, limits, relative)
    return x, w/np.sum(w)
