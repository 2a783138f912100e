"""
SAS-flop totals of the measured configurations (measurement
infrastructure: the roofline numerator; never on the product path).

Runs the counting restatement built by ``oracle/build_oracle.py``
(``oracle/_build/libsasflops_<model>.so``): the reference's own model C
compiled with a counting arithmetic type, on the configuration's own
marshaled inputs, so that every branch the reference takes is replayed and
the operations of the branches taken are counted under the "SAS-flop v1"
convention (see oracle/sasflops.hpp).

    python oracle/sasflops.py [sphere1d cylinder2d magnetic ...] [--threads N]

prints one JSON object per configuration: SAS-flops per evaluation (the
mean over the configuration), per mesh point and per q point, the totals,
and the branch mix (how many evaluations cost how many SAS-flops).
"""

import argparse
import ctypes as ct
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

_LIBS = {}


def _lib(name):
    if name not in _LIBS:
        path = os.path.join(HERE, "_build", "libsasflops_%s.so" % name)
        if not os.path.exists(path):
            raise RuntimeError("SAS-flop counter for %s not built (%s); run "
                               "python oracle/build_oracle.py" % (name, path))
        lib = ct.CDLL(path)
        fn = lib.sasflops_count
        fn.argtypes = [ct.c_int, ct.c_int32, ct.c_void_p, ct.c_void_p, ct.c_int32,
                       ct.c_void_p, ct.c_double, ct.c_int32, ct.c_int, ct.c_void_p,
                       ct.c_void_p, ct.c_int32]
        fn.restype = ct.c_int
        _LIBS[name] = fn
    return _LIBS[name]


def threads_available():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def count(name, q_vectors, pars, cutoff=0.0, reff_mode=0, threads=None, nbins=4096):
    """SAS-flops of one kernel call of model *name* at *q_vectors* with the
    parameter dict *pars* (dispersity given as name_pd, name_pd_n, ...).
    Returns a dict of the three buckets, the evaluation count and the branch
    mix {SAS-flops per evaluation: evaluations}."""
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.details import make_kernel_args
    from sasmodels_b200.direct_model import get_mesh
    info = load_model_info(name)
    dim = '2d' if len(q_vectors) == 2 else '1d'

    class _Shape:
        pass
    shape = _Shape()
    shape.info, shape.dim, shape.dtype = info, dim, np.dtype('d')
    pars = dict(pars)
    pars.pop("radius_effective_mode", None)
    details, values, magnetic = make_kernel_args(shape, get_mesh(info, pars, dim=dim))
    variant = 0 if dim == '1d' else (2 if magnetic else 1)
    if dim == '1d':
        q = np.ascontiguousarray(q_vectors[0], 'd')
    else:
        q = np.empty(2*len(q_vectors[0]), 'd')
        q[0::2], q[1::2] = q_vectors
    nq = len(q_vectors[0])
    buf = np.ascontiguousarray(details.buffer, np.int32)
    values = np.ascontiguousarray(values, 'd')
    totals = np.zeros(5, np.uint64)
    hist = np.zeros(nbins, np.uint64)
    rc = _lib(name)(variant, nq, buf.ctypes.data, values.ctypes.data, values.size,
                    q.ctypes.data, float(cutoff), int(reff_mode),
                    int(threads or threads_available()), totals.ctypes.data,
                    hist.ctypes.data, nbins)
    if rc != 0:
        raise RuntimeError("sasflops_count(%s) returned %d" % (name, rc))
    evals = int(totals[3])
    mix = {int(c): int(n) for c, n in zip(np.nonzero(hist)[0], hist[np.nonzero(hist)[0]])}
    if hist[-1]:
        mix["overflow(>=%d)" % (nbins - 1)] = mix.pop(nbins - 1)
    return {"model": name, "variant": ["Iq", "Iqxy", "Imagnetic"][variant],
            "nq": nq, "mesh_points": int(details.num_eval), "kept_points": int(totals[4]),
            "evals": evals, "eval_sasflops": int(totals[0]),
            "point_sasflops": int(totals[1]), "q_sasflops": int(totals[2]),
            "total_sasflops": int(totals[0] + totals[1] + totals[2]),
            "sasflops_per_eval": float(totals[0])/evals if evals else 0.0,
            "sasflops_per_eval_all_in": (float(totals[0] + totals[1] + totals[2])/evals
                                         if evals else 0.0),
            "branch_mix": mix}


def config(name, threads=None):
    """SAS-flops of a headline configuration at its full size."""
    from sasmodels_b200 import workloads
    if name == "sphere1d":
        model, qv, pars = workloads.sphere_1d()
    elif name == "cylinder2d":
        model, qv, pars = workloads.cylinder_2d()
    elif name == "magnetic":
        model, qv, pars = workloads.core_shell_sphere_magnetic()
    elif name.startswith("cylinder2d_strided"):
        model, qv, pars = workloads.cylinder_2d_strided(int(name.rsplit("_", 1)[1]))
    else:
        raise ValueError(name)
    t0 = time.time()
    out = count(model, qv, pars, threads=threads)
    out["config"] = name
    out["count_seconds"] = round(time.time() - t0, 1)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("configs", nargs="*", default=["sphere1d", "magnetic", "cylinder2d"])
    ap.add_argument("--threads", type=int, default=None)
    args = ap.parse_args(argv)
    for name in args.configs:
        print(json.dumps(config(name, args.threads)), flush=True)


if __name__ == "__main__":
    main()
