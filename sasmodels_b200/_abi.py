"""
ctypes binding of the per-model C-ABI (include/sasb200.h).

Every symbol takes device pointers and a CUDA stream handle; nothing here
allocates or copies.  A missing or unloadable library raises RuntimeError:
there is no CPU fallback on the product path.
"""

import ctypes as ct
import json
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

VARIANTS = ("Iq", "Iqxy", "Imagnetic")
VARIANT_ID = {name: k for k, name in enumerate(VARIANTS)}

_KERNEL_ARGTYPES = [
    ct.c_int32, ct.c_int32, ct.c_int32,      # nq, pd_start, pd_stop
    ct.c_void_p, ct.c_void_p, ct.c_void_p,   # details, values, q
    ct.c_void_p,                             # result
    ct.c_double, ct.c_int32,                 # cutoff, radius_effective_mode
    ct.c_void_p, ct.c_uint64,                # workspace, workspace_bytes
    ct.c_int32, ct.c_void_p,                 # tile, stream
]

_LOADED = {}


def library_path(name, lib_dir=None):
    return os.path.join(lib_dir or LIB_DIR, "libsasb200_%s.so" % name)


def metadata_path(name, lib_dir=None):
    return os.path.join(lib_dir or LIB_DIR, "%s.json" % name)


def available_models(lib_dir=None):
    d = lib_dir or LIB_DIR
    if not os.path.isdir(d):
        return []
    return sorted(f[len("libsasb200_"):-3] for f in os.listdir(d)
                  if f.startswith("libsasb200_") and f.endswith(".so")
                  and os.path.exists(os.path.join(d, f[len("libsasb200_"):-3] + ".json")))


class ModelLib:
    """The exported functions of one ``libsasb200_<model>.so`` under one
    symbol prefix: ``<model>`` for the FP64 form, ``<model>_f32c`` for the
    FP32-compensated form of the same library."""

    def __init__(self, name, path=None):
        self.name = name
        self.path = path or library_path(name)
        if not os.path.exists(self.path):
            raise RuntimeError(
                "B200 library for model %r not found at %s; run "
                "`python -m sasmodels_b200.build %s`" % (name, self.path, name))
        try:
            self.lib = ct.CDLL(self.path)
        except OSError as exc:
            raise RuntimeError("cannot load %s: %s" % (self.path, exc)) from exc
        self.kernels = {}
        for variant in VARIANTS:
            fn = getattr(self.lib, "sasb200_%s_%s" % (name, variant))
            fn.argtypes = _KERNEL_ARGTYPES
            fn.restype = ct.c_int32
            self.kernels[variant] = fn
        self._ws = self._fn("workspace_bytes", ct.c_uint64,
                            [ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32])
        self._err = self._fn("last_error", ct.c_char_p, [])
        self._ntile = self._fn("tile_count", ct.c_int32, [])
        self._tile = self._fn("tile_code", ct.c_int32, [ct.c_int32])
        self._default_tile = self._fn("default_tile", ct.c_int32,
                                      [ct.c_int32, ct.c_int32, ct.c_int32])
        self._single_max = self._fn("single_launch_max", ct.c_int32, [ct.c_int32])

    def _fn(self, suffix, restype, argtypes):
        fn = getattr(self.lib, "sasb200_%s_%s" % (self.name, suffix))
        fn.restype = restype
        fn.argtypes = argtypes
        return fn

    def workspace_bytes(self, variant, nq, n_mesh, tile=0):
        return int(self._ws(VARIANT_ID[variant], nq, n_mesh, tile))

    def last_error(self):
        msg = self._err()
        return msg.decode() if msg else ""

    def tile_shapes(self):
        return [int(self._tile(i)) for i in range(int(self._ntile()))]

    def default_tile(self, variant, nq, n_mesh):
        return int(self._default_tile(VARIANT_ID[variant], nq, n_mesh))

    def single_launch_max(self, variant):
        """Largest mesh range the library evaluates in one kernel launch."""
        return int(self._single_max(VARIANT_ID[variant]))

    def launches(self, variant, nq, n_mesh, workspace_bytes=None, tile=0):
        """Kernel launches of one call over a mesh range of n_mesh points
        (1 on the single-launch path, else 3 per workspace chunk)."""
        if n_mesh <= self.single_launch_max(variant):
            return 1
        full = self.workspace_bytes(variant, nq, n_mesh, tile)
        if workspace_bytes is None or workspace_bytes >= full:
            return 3*max(1, -(-n_mesh//(1 << 20)))
        return 3*max(1, -(-full//max(workspace_bytes, 1)))

    def call(self, variant, nq, pd_start, pd_stop, details, values, q, result,
             cutoff, reff_mode, workspace, workspace_bytes, tile, stream):
        status = self.kernels[variant](
            nq, pd_start, pd_stop, details, values, q, result, cutoff,
            reff_mode, workspace, workspace_bytes, tile, stream)
        if status != 0:
            raise RuntimeError("sasb200_%s_%s failed (%d): %s" % (
                self.name, variant, status, self.last_error()))


#: symbol prefix of each form within a model's library: the FP64 form, the
#: FP32-compensated form, and (for models with a hoisted FP64 binding) the
#: plugin's C as translated, without the hoisting
FORM_PREFIX = {"double": "%s", "float32c": "%s_f32c", "plugin": "%s_plugin"}


def load_library(name, lib_dir=None, form="double"):
    """Entry points of model *name*; *form* is "double", "float32c" or
    "plugin"."""
    key = (name, lib_dir, form)
    if key not in _LOADED:
        if form not in FORM_PREFIX:
            raise ValueError("unknown form %r" % (form,))
        _LOADED[key] = ModelLib(FORM_PREFIX[form] % name, library_path(name, lib_dir))
    return _LOADED[key]


def load_metadata(name, lib_dir=None):
    path = metadata_path(name, lib_dir)
    if not os.path.exists(path):
        raise RuntimeError("no B200 metadata for model %r at %s" % (name, path))
    with open(path) as fid:
        return json.load(fid)
