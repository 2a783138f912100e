"""
Caller for the reference DLL oracle in ``oracle/_ref`` (test infrastructure).

Only tests, the smoke check and the CPU-baseline leg of the benchmark use
this module; the product path never does.

The DLL symbols have the reference signature (``sasmodels/kernel_iq.c:317-328``,
ctypes argtypes ``sasmodels/kerneldll.py:368-375``) and are called the way
``DllKernel._call_kernel`` does (``kerneldll.py:449-475``): in chunks of 100
mesh points, with the result buffer carrying the partial sums between
chunks.  :func:`run_threads` shards q across host threads, one independent
call per thread on a disjoint q slice (ctypes releases the GIL), which gives
bitwise the same numbers as one thread.
"""

import ctypes as ct
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_ARGTYPES = [ct.c_int32]*3 + [ct.c_void_p]*4 + [ct.c_double, ct.c_int32]
_LIBS = {}


def ref_path(name):
    return os.path.join(REF_DIR, "sas64_%s.so" % name)


def available(name):
    return os.path.exists(ref_path(name))


class RefDll:
    """The three exported kernels of one reference model DLL."""

    def __init__(self, name):
        path = ref_path(name)
        if not os.path.exists(path):
            raise RuntimeError("reference DLL for %s not built (%s); run "
                               "python oracle/build_ref.py" % (name, path))
        self.name = name
        self.lib = ct.CDLL(path)
        self.fns = {}
        for variant in ("Iq", "Iqxy", "Imagnetic"):
            fn = self.lib["%s_%s" % (name, variant)]
            fn.argtypes = _ARGTYPES
            fn.restype = None
            self.fns[variant] = fn

    def call(self, variant, q, details, values, nout, cutoff=0.0,
             reff_mode=0, step=100, pd_start=0, pd_stop=None, result=None):
        """
        Evaluate the reference kernel.  *q* is the 1D q vector or the
        interleaved (qx, qy) array; *nout* is 2 for 1D Fq models else 1.
        Returns the raw result vector (nout*nq values + 4 norms).
        """
        q = np.ascontiguousarray(q, 'd')
        nq = q.size//2 if variant != "Iq" else q.size
        details = np.ascontiguousarray(details, np.int32)
        values = np.ascontiguousarray(values, 'd')
        if result is None:
            result = np.zeros(nout*nq + 4, 'd')
        num_eval = int(details[-4]) if pd_stop is None else pd_stop
        fn = self.fns[variant]
        start = pd_start
        while True:
            stop = min(start + step, num_eval)
            fn(nq, start, stop, details.ctypes.data, values.ctypes.data,
               q.ctypes.data, result.ctypes.data, cutoff, reff_mode)
            start = stop
            if start >= num_eval:
                break
        return result


def load(name):
    if name not in _LIBS:
        _LIBS[name] = RefDll(name)
    return _LIBS[name]


def run_threads(name, variant, q, details, values, nout, threads, cutoff=0.0,
                reff_mode=0):
    """q-sharded multi-thread evaluation; returns the same result vector
    as a single call."""
    dll = load(name)
    q = np.ascontiguousarray(q, 'd')
    per = 2 if variant != "Iq" else 1
    nq = q.size//per
    threads = max(1, min(threads, nq))
    bounds = np.linspace(0, nq, threads + 1).astype(int)

    def part(k):
        lo, hi = bounds[k], bounds[k+1]
        return dll.call(variant, q[lo*per:hi*per], details, values, nout,
                        cutoff, reff_mode)

    with ThreadPoolExecutor(max_workers=threads) as pool:
        parts = list(pool.map(part, range(threads)))
    out = np.empty(nout*nq + 4, 'd')
    for k, res in enumerate(parts):
        lo, hi = bounds[k], bounds[k+1]
        out[nout*lo:nout*hi] = res[:nout*(hi-lo)]
    out[nout*nq:] = parts[0][-4:]
    return out


def run_mesh_threads(name, variant, q, details, values, nout, threads, cutoff=0.0,
                     reff_mode=0):
    """Mesh-sharded multi-thread evaluation for calls with few q points and a
    large dispersity mesh: thread k evaluates the contiguous mesh range
    [pd_start_k, pd_stop_k) into its own zeroed result (the reference's
    restart contract, kernel_iq.c:381-423), and the partial vectors are added
    in range order.  Equal to one call up to the rounding of those adds
    (far below the 1e-12 bar)."""
    dll = load(name)
    details = np.ascontiguousarray(details, np.int32)
    num_eval = int(details[-4])
    threads = max(1, min(threads, num_eval))
    bounds = np.linspace(0, num_eval, threads + 1).astype(int)
    per = 2 if variant != "Iq" else 1
    nq = np.asarray(q).size//per

    def part(k):
        res = np.zeros(nout*nq + 4, 'd')
        if bounds[k] == bounds[k+1]:
            return res
        return dll.call(variant, q, details, values, nout, cutoff, reff_mode,
                        pd_start=int(bounds[k]), pd_stop=int(bounds[k+1]), result=res)

    with ThreadPoolExecutor(max_workers=threads) as pool:
        parts = list(pool.map(part, range(threads)))
    out = parts[0].copy()
    for res in parts[1:]:
        out += res
    return out
