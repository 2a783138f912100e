"""
Dispersity distributions: parameter value -> (mesh values, normalised weights).

Same distributions, defaults and truncation rules as the sasmodels plugin API
(``sasmodels/weights.py``): the kernels consume the weight vectors these
produce, so the points and weights must be identical for the DLL and the B200
path to integrate over the same mesh.
"""

from collections import OrderedDict

import numpy as np
from scipy.special import gammaln


class Dispersion:
    """Base distribution (``weights.py:21-83``)."""
    type = "base disperser"
    default = dict(npts=35, width=0, nsigmas=3)

    def __init__(self, npts=None, width=None, nsigmas=None):
        self.npts = self.default['npts'] if npts is None else int(npts)
        self.width = self.default['width'] if width is None else width
        self.nsigmas = self.default['nsigmas'] if nsigmas is None else nsigmas

    def get_weights(self, center, lb, ub, relative):
        """
        Values and (unnormalised) weights.  Volume parameters use a width
        relative to *center*; orientation jitter is absolute and centred on
        zero (``weights.py:50-72``).
        """
        sigma = self.width*center if relative else self.width
        if not relative:
            center = 0
        if sigma == 0 or self.npts < 2:
            if lb <= center <= ub:
                return np.array([center], 'd'), np.array([1.], 'd')
            return np.array([], 'd'), np.array([], 'd')
        return self._weights(center, sigma, lb, ub)

    def _weights(self, center, sigma, lb, ub):
        raise NotImplementedError

    def _linspace(self, center, sigma, lb, ub):
        """npts evenly spaced over +/- nsigmas, clipped to [lb, ub]
        (``weights.py:78-83``)."""
        x = center + np.linspace(-self.nsigmas*sigma, +self.nsigmas*sigma,
                                 self.npts)
        return x[(x >= lb) & (x <= ub)]


class GaussianDispersion(Dispersion):
    """``weights.py:86-102``"""
    type = "gaussian"
    default = dict(npts=35, width=0, nsigmas=3)

    def _weights(self, center, sigma, lb, ub):
        x = self._linspace(center, sigma, lb, ub)
        return x, np.exp((x-center)**2 / (-2.0*sigma*sigma))


class UniformDispersion(Dispersion):
    """``weights.py:104-117``"""
    type = "uniform"
    default = dict(npts=35, width=0, nsigmas=None)

    def _weights(self, center, sigma, lb, ub):
        x = np.linspace(center-sigma, center+sigma, self.npts)
        x = x[(x >= lb) & (x <= ub)]
        return x, np.ones_like(x)


class RectangleDispersion(Dispersion):
    """``weights.py:119-132``"""
    type = "rectangle"
    default = dict(npts=35, width=0, nsigmas=1.73205)

    def _weights(self, center, sigma, lb, ub):
        x = self._linspace(center, sigma, lb, ub)
        x = x[np.fabs(x-center) <= np.fabs(sigma)*np.sqrt(3.0)]
        return x, np.ones_like(x)


class LogNormalDispersion(Dispersion):
    """``weights.py:134-149``"""
    type = "lognormal"
    default = dict(npts=80, width=0, nsigmas=8)

    def _weights(self, center, sigma, lb, ub):
        x = self._linspace(center, sigma, max(lb, 1e-8), max(ub, 1e-8))
        sig = np.fabs(sigma/center)
        px = np.exp(-0.5*((np.log(x)-np.log(center))/sig)**2)/(x*sig)
        return x, px


class SchulzDispersion(Dispersion):
    """``weights.py:152-176``"""
    type = "schulz"
    default = dict(npts=80, width=0, nsigmas=8)

    def _weights(self, center, sigma, lb, ub):
        x = self._linspace(center, sigma, max(lb, 1e-8), max(ub, 1e-8))
        R = x/center
        z = (center/sigma)**2
        arg = z*np.log(z) + (z-1)*np.log(R) - R*z - np.log(center) - gammaln(z)
        return x, np.exp(arg)


class ArrayDispersion(Dispersion):
    """``weights.py:179-205``"""
    type = "array"
    default = dict(npts=35, width=0, nsigmas=1)

    def __init__(self, npts=None, width=None, nsigmas=None):
        Dispersion.__init__(self, npts, width, nsigmas)
        self.values = np.array([0.], 'd')
        self.weights = np.array([1.], 'd')

    def set_weights(self, values, weights):
        self.values = np.ascontiguousarray(values, 'd')
        self.weights = np.ascontiguousarray(weights, 'd')
        self.npts = len(values)

    def _weights(self, center, sigma, lb, ub):
        idx = (self.values >= lb) & (self.values <= ub)
        return self.values[idx], self.weights[idx]


class BoltzmannDispersion(Dispersion):
    """``weights.py:207-220``"""
    type = "boltzmann"
    default = dict(npts=35, width=0, nsigmas=3)

    def _weights(self, center, sigma, lb, ub):
        x = self._linspace(center, sigma, lb, ub)
        return x, np.exp(-np.abs(x-center) / np.abs(sigma))


#: name -> distribution class, in the order sasview lists them
#: (``weights.py:225-233``).
DISTRIBUTIONS = OrderedDict((d.type, d) for d in (
    RectangleDispersion,
    UniformDispersion,
    ArrayDispersion,
    LogNormalDispersion,
    GaussianDispersion,
    SchulzDispersion,
    BoltzmannDispersion,
))
MODELS = DISTRIBUTIONS


def get_weights(disperser, n, width, nsigmas, value, limits, relative):
    """
    (values, weights) for one polydisperse parameter with weights normalised
    to sum to one (``weights.py:264-291``).
    """
    if disperser == "array":
        raise NotImplementedError("Don't handle arrays through get_weights;"
                                  " use values and weights directly")
    cls = DISTRIBUTIONS[disperser]
    obj = cls(n, width, nsigmas)
    v, w = obj.get_weights(value, limits[0], limits[1], relative)
    return v, w/np.sum(w)
