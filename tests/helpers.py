"""Shared test helpers: marshaling through the host mirror, the reference
DLL oracle, normalisation and the comparison rules used by the tests."""

import json
import os

import numpy as np

from sasmodels_b200 import core
from sasmodels_b200.details import make_kernel_args
from sasmodels_b200.direct_model import RADIUS_MODE_ID, get_mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODELS = ["sphere", "cylinder", "core_shell_sphere", "ellipsoid",
          "core_shell_cylinder"]

#: FP64 parity bar against the reference DLL on identical inputs
RTOL_FP64 = 1e-12


def golden(name):
    with open(os.path.join(GOLDEN, "%s.json" % name)) as fid:
        return json.load(fid)


class HostKernel:
    """Just enough of a Kernel for make_kernel_args (info, dim, dtype)."""
    def __init__(self, info, dim):
        self.info = info
        self.dim = dim
        self.dtype = np.dtype('d')


def marshal(info, pars, q_vectors, mono=False):
    dim = '2d' if len(q_vectors) == 2 else '1d'
    pars = dict(pars)
    pars.pop(RADIUS_MODE_ID, None)
    mesh = get_mesh(info, pars, dim=dim, mono=mono)
    details, values, magnetic = make_kernel_args(HostKernel(info, dim), mesh)
    return details, values, magnetic


def interleave(q_vectors):
    if len(q_vectors) == 1:
        return np.ascontiguousarray(q_vectors[0], 'd')
    q = np.empty(2*len(q_vectors[0]), 'd')
    q[0::2] = q_vectors[0]
    q[1::2] = q_vectors[1]
    return q


def variant(dim, magnetic):
    return "Iq" if dim == '1d' else ("Imagnetic" if magnetic else "Iqxy")


def nout_of(info, dim):
    return 2 if info.have_Fq and dim == '1d' else 1


def reference_raw(name, info, q_vectors, pars, cutoff=0.0, reff_mode=0, threads=1):
    from oracle import refdll
    details, values, magnetic = marshal(info, pars, q_vectors)
    dim = '2d' if len(q_vectors) == 2 else '1d'
    nout = nout_of(info, dim)
    q = interleave(q_vectors)
    if threads > 1:
        return refdll.run_threads(name, variant(dim, magnetic), q, details.buffer,
                                  values, nout, threads, cutoff, reff_mode)
    return refdll.load(name).call(variant(dim, magnetic), q, details.buffer,
                                  values, nout, cutoff, reff_mode)


def normalise(raw, nout, nq, values):
    """Kernel.Fq/Iq arithmetic (sasmodels/kernel.py:80-188) on a raw vector."""
    total = raw[nout*nq]
    if total == 0.:
        total = 1.
    form = raw[nout*nq + 1]/total
    shell = raw[nout*nq + 2]/total
    reff = raw[nout*nq + 3]/total
    if shell == 0.:
        shell = 1.
    F1 = raw[1:nout*nq:nout]/total if nout == 2 else None
    F2 = raw[0:nout*nq:nout]/total
    I = values[0]/shell*F2 + values[1]
    return dict(F1=F1, F2=F2, reff=reff, shell=shell, ratio=form/shell, I=I)


def is_near(target, actual, digits=5):
    """Significant-digit match of sasmodels/model_test.py:443-471."""
    if target is None:
        return not np.isnan(actual)
    if target == 0.:
        return actual == 0.
    if np.isfinite(target):
        shift = np.ceil(np.log10(abs(target)))
        return abs(target - actual) < 1.5*10**(shift - digits)
    if target == actual:
        return True
    return np.isnan(target) == np.isnan(actual)


def compare_raw(ours, ref, nout, nq, rtol=RTOL_FP64):
    """
    Max error of a raw result vector against the reference, in units of the
    tolerance scale of each slot:

    * F^2 slots and the four norms: relative to |ref|;
    * F slots (<F> can cross zero): relative to sqrt(sum(w) * <F^2> sum),
      the Cauchy-Schwarz bound on |<F>| sum, so a zero crossing of <F> does
      not turn rounding noise into an unbounded relative error.

    Returns (worst ratio err/(rtol*scale), worst relative F^2 error).
    """
    ours = np.asarray(ours, 'd')
    ref = np.asarray(ref, 'd')
    err = np.abs(ours - ref)
    scale = np.abs(ref).copy()
    if nout == 2:
        f2 = np.abs(ref[0:2*nq:2])
        scale[1:2*nq:2] = np.sqrt(f2*abs(ref[2*nq]))
    tiny = np.finfo(float).tiny
    ratio = err/np.maximum(rtol*scale, tiny)
    ratio[(err == 0)] = 0.0
    f2_rel = err[0:nout*nq:nout]/np.maximum(np.abs(ref[0:nout*nq:nout]), tiny)
    f2_rel[err[0:nout*nq:nout] == 0] = 0.0
    return float(ratio.max(initial=0.0)), float(f2_rel.max(initial=0.0))


def load_info(name):
    return core.load_model_info(name)
