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


def reference_raw(name, info, q_vectors, pars, cutoff=0.0, reff_mode=0, threads=1,
                  split="q"):
    """Raw result vector of the reference DLL.  With threads > 1 the call is
    sharded over host threads by q (bitwise equal to one call) or, with
    split="mesh", by dispersity-mesh range (for few q and a large mesh)."""
    from oracle import refdll
    details, values, magnetic = marshal(info, pars, q_vectors)
    dim = '2d' if len(q_vectors) == 2 else '1d'
    nout = nout_of(info, dim)
    q = interleave(q_vectors)
    if threads > 1 and split == "mesh":
        return refdll.run_mesh_threads(name, variant(dim, magnetic), q, details.buffer,
                                       values, nout, threads, cutoff, reff_mode)
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


def host_threads():
    """Host threads this process may use (for sharding oracle calls)."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


#: members of the 4096-set seeded fit population (workloads.population,
#: seed 1) at full size, with the q points of each set that the parity tests
#: evaluate (indices into the set's own q vector; each q is independent):
#:   1747 core_shell_cylinder, pd 67 x 59 x 68 = 268,804 points; its largest
#:        q puts 50,451 (q, mesh point) pairs on the 5000-point Gauss rule
#:   2975 core_shell_cylinder, pd 65 x 66 x 67 = 287,430 points
#:   3    core_shell_cylinder, pd 55 x 66 x 62 = 225,060 points
#:   563  core_shell_cylinder, pd 39 on one dimension, 5000-point rule at top q
#:   924  ellipsoid, pd 65 x 63, 500-point rule at top q
#:   2584 ellipsoid, pd 71 x 60
FULL_SIZE_SETS = {1747: 3, 2975: 3, 3: 6, 563: 12, 924: 12, 2584: 12}


def full_size_population():
    """[(index, model, q_subsample, pars)] of FULL_SIZE_SETS: each set's
    full dispersity mesh at its smallest, largest and evenly spaced q."""
    import numpy as np
    from sasmodels_b200 import workloads
    pop = workloads.population(n_sets=4096, seed=1)
    out = []
    for k, nsub in FULL_SIZE_SETS.items():
        name, q, pars = pop[k]
        idx = np.unique(np.linspace(0, len(q) - 1, nsub).round().astype(int))
        out.append((k, name, q[idx], pars))
    return out


_FULL_SIZE_REF = {}


def full_size_reference(k, name, q, pars):
    """Reference DLL raw vector of a FULL_SIZE_SETS member (mesh-sharded over
    the host threads), computed once per process."""
    if k not in _FULL_SIZE_REF:
        _FULL_SIZE_REF[k] = reference_raw(name, load_info(name), [q], pars,
                                          threads=host_threads(), split="mesh")
    return _FULL_SIZE_REF[k]


def gauss_rule_counts(name, q, pars):
    """{rule length: number of (q, mesh point) pairs} for a 1D ellipsoid or
    core_shell_cylinder call: the adaptive Gauss rule each pair uses, chosen
    from q times the largest dimension of that mesh point
    (models/lib/adaptive.c gauss_weights; models/ellipsoid.c,
    models/core_shell_cylinder.c)."""
    import numpy as np
    from sasmodels_b200.batch import rule_points
    info = load_info(name)
    mesh = {p.name: np.asarray(m[1]) for p, m in
            zip(info.parameters.call_parameters, get_mesh(info, pars, dim='1d'))}
    if name == "ellipsoid":
        r = np.maximum.outer(mesh["radius_polar"], mesh["radius_equatorial"]).ravel()
    else:
        r = np.maximum(np.add.outer(mesh["radius"], mesh["thickness"])[:, :, None],
                       (0.5*mesh["length"])[None, None, :]
                       + mesh["thickness"][None, :, None]).ravel()
    n = rule_points(np.outer(q, r))
    return {int(k): int((n == k).sum()) for k in (20, 76, 500, 5000)}
