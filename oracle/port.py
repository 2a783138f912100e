"""
Caller for the CPU restatement oracle (oracle/sas_oracle.c, built by
oracle/build_oracle.py into oracle/_build).  Test infrastructure only.
"""

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
_VARIANT = {"Iq": 0, "Iqxy": 1, "Imagnetic": 2}
_LIBS = {}


def lib_path(name):
    return os.path.join(BUILD, "liboracle_%s.so" % name)


class OraclePort:
    def __init__(self, name):
        path = lib_path(name)
        if not os.path.exists(path):
            raise RuntimeError("oracle restatement for %s not built (%s); run "
                               "python oracle/build_oracle.py" % (name, path))
        self.lib = ct.CDLL(path)
        fn = self.lib.oracle_kernel
        fn.argtypes = [ct.c_int, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_void_p,
                       ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_double,
                       ct.c_int32, ct.c_int]
        fn.restype = ct.c_int
        self.fn = fn

    def call(self, variant, q, details, values, nout, cutoff=0.0, reff_mode=0,
             threads=1, pd_start=0, pd_stop=None, result=None):
        q = np.ascontiguousarray(q, 'd')
        nq = q.size//2 if variant != "Iq" else q.size
        details = np.ascontiguousarray(details, np.int32)
        values = np.ascontiguousarray(values, 'd')
        if result is None:
            result = np.zeros(nout*nq + 4, 'd')
        stop = int(details[-4]) if pd_stop is None else pd_stop
        status = self.fn(_VARIANT[variant], nq, pd_start, stop, details.ctypes.data,
                         values.ctypes.data, q.ctypes.data, result.ctypes.data,
                         cutoff, reff_mode, threads)
        if status != 0:
            raise RuntimeError("oracle_kernel failed (%d)" % status)
        return result


def load(name):
    if name not in _LIBS:
        _LIBS[name] = OraclePort(name)
    return _LIBS[name]
