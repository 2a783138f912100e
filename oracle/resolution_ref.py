"""
CPU restatement of the reference's resolution smearing (test infrastructure
only: tests use it as the checker; the product never imports it).

* pinhole_matrix / smear_1d: the dense n_calc x nq pinhole weight matrix
  (gaussian bin masses from erf at the bin edges, cut to [q - 2.5 s,
  q + 3 s], columns normalised) and theory . W
  (sasmodels/resolution.py:172-220, bin edges :423-438);
* slit_matrix: the slit weights (u-substituted bin widths between |q| and
  sqrt(q^2 + l^2), averaged over 2 n + 1 steps across the width;
  sasmodels/resolution.py:223-395);
* average_2d: the weighted average over the oversampling bins of each 2D
  point (sasmodels/resolution2d.py:162-175).

Pinned by tests/golden/resolution.json, produced by the reference itself
(tests/golden/make_resolution_golden.py).
"""

import numpy as np
from scipy.special import erf


def bin_edges(x):
    return np.hstack([x[0] - 0.5*(x[1] - x[0]), 0.5*(x[1:] + x[:-1]),
                      x[-1] + 0.5*(x[-1] - x[-2])])


def pinhole_matrix(q_calc_signed, q, q_width, nsigma=(2.5, 3.0)):
    """Weights W[j, i] of calculated point j in measured point i."""
    edges = bin_edges(q_calc_signed)
    cdf = erf((edges[:, None] - q[None, :])/(np.sqrt(2.0)*q_width)[None, :])
    w = cdf[1:] - cdf[:-1]
    lo, hi = nsigma
    w[q_calc_signed[:, None] < (q - lo*q_width)[None, :]] = 0.
    w[q_calc_signed[:, None] > (q + hi*q_width)[None, :]] = 0.
    w /= np.sum(w, axis=0)[None, :]
    return w


def smear_1d(weight_matrix, theory):
    return np.dot(theory[None, :], weight_matrix).flatten()


def average_2d(theory, weights, nq):
    nbins = len(weights)
    return np.average(np.reshape(theory, (nbins, nq)), axis=0, weights=weights)


def _perp(edges, qi, length):
    limit = np.sqrt(qi**2 + length**2)
    u = edges**2 - qi**2
    u[edges < abs(qi)] = 0.
    u[edges > limit] = limit**2 - qi**2
    return np.diff(np.sqrt(u))/length


def slit_matrix(q_calc_signed, q, q_length, q_width, n_length=30):
    """W[j, i]: weight of calculated point j in measured point i."""
    edges = bin_edges(q_calc_signed)
    w = np.zeros((len(q), len(q_calc_signed)))
    for i, (qi, wi, li) in enumerate(zip(q, q_width, q_length)):
        if wi == 0. and li == 0.:
            w[i, :] = (q_calc_signed == qi)
        elif wi == 0:
            w[i, :] = _perp(edges, qi, li)
        else:
            for k in range(-n_length, n_length + 1):
                w[i, :] += _perp(edges, qi + k*wi/n_length, li)
            w[i, :] /= 2*n_length + 1
    return w.T
