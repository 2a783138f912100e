"""
Model loading for the B200 backend, mirroring ``sasmodels/core.py``
(``load_model`` 117-128, ``load_model_info`` 130-169, ``build_model``
293-341).

``load_model("cylinder")`` works from the prebuilt library and its JSON
metadata alone.  ``build_model(info)`` also accepts a sasmodels
``ModelInfo`` (and compiles the library if it is missing, which needs
sasmodels' model sources and nvcc).  :func:`install` routes
``sasmodels.core.build_model(..., platform="b200")`` here so existing
callers (``direct_model``, ``bumps_model``, ``sasview_model``, product and
mixture kernels) pick up the B200 engine without edits.
"""

import os

from . import _abi
from .kernel import B200Model
from .modelinfo import ModelInfo

PLATFORM = "b200"


def list_models():
    """Models with a built B200 library."""
    return _abi.available_models()


def load_model_info(name, lib_dir=None):
    """Our :class:`ModelInfo` from the JSON written beside the library;
    ``"P@S"`` names give the product info (``core.py:130-169``)."""
    if "@" in name:
        from .product import make_product_info
        p_name, s_name = name.split("@", 1)
        return make_product_info(load_model_info(p_name, lib_dir),
                                 load_model_info(s_name, lib_dir))
    return ModelInfo(_abi.load_metadata(name, lib_dir))


def load_model(name, dtype="double", platform=PLATFORM, device=None):
    """Engine for model *name* (``core.py:117-128``)."""
    if platform != PLATFORM:
        raise ValueError("sasmodels_b200 only provides platform %r" % PLATFORM)
    return build_model(load_model_info(name), dtype=dtype, device=device)


def build_model(model_info, dtype=None, platform=PLATFORM, device=None):
    """Engine for *model_info*, ours or a sasmodels ModelInfo (``core.py:293-341``).

    A sasmodels ModelInfo stays the engine's ``info`` (what the reference's
    callers read back); this backend's own description of the model, from
    the library's metadata, drives the engine."""
    if platform not in (PLATFORM, None):
        raise ValueError("sasmodels_b200 only provides platform %r" % PLATFORM)
    info = model_info
    composition = getattr(info, "composition", None)
    if composition and composition[0] == "product":
        from .product import B200ProductModel, make_product_info
        p_info, s_info = composition[1]
        P = build_model(p_info, dtype=dtype, device=device)
        S = build_model(s_info, dtype=dtype, device=device)
        if not isinstance(info, ModelInfo):
            info = make_product_info(P.meta, S.meta)
        return B200ProductModel(info, P, S)
    if composition:
        raise ValueError("sasmodels_b200 builds products (P@S) itself; build %r "
                         "mixtures through sasmodels.core.build_model after install()"
                         % getattr(info, "id", info))
    if not isinstance(info, ModelInfo):
        name = info.id
        if name not in _abi.available_models():
            from . import build
            build.build_model(name)
        return B200Model(info, dtype=dtype, device=device, meta=load_model_info(name))
    return B200Model(info, dtype=dtype, device=device)


_ORIGINAL = {}


def routes_here(platform):
    """True if a ``sasmodels.core.build_model`` call with *platform* goes to
    this backend: ``platform="b200"``, or the default platform with
    ``SAS_OPENCL=b200`` in the environment."""
    env = os.environ.get("SAS_OPENCL", "").lower()
    return platform == PLATFORM or (platform == "ocl" and env == PLATFORM)


def install():
    """
    Route ``sasmodels.core.build_model(info, dtype, platform="b200")`` (and
    ``SAS_OPENCL=b200``) to this backend.  The reference package is left
    untouched on disk; only the function object in its module is wrapped, so
    ``load_model`` and the recursive builds of compositions inside
    ``sasmodels.core`` go through the wrapper too.  Mixtures stay the
    reference's ``MixtureModel`` over B200 parts; pure-Python models stay
    the reference's; products (P@S) run on the device here.
    """
    import sasmodels.core as sc
    if "build_model" in _ORIGINAL:
        return
    original = sc.build_model
    _ORIGINAL["build_model"] = original

    def build_model_b200(model_info, dtype=None, platform="ocl"):
        if routes_here(platform):
            composition = getattr(model_info, "composition", None)
            mixture = composition is not None and composition[0] == "mixture"
            if mixture or not getattr(model_info, "compiled", True):
                # the reference's own MixtureModel (its parts come back
                # through this wrapper) or its pure-Python kernel
                return original(model_info, dtype=dtype,
                                platform="dll" if not mixture else platform)
            return build_model(model_info, dtype=dtype)
        return original(model_info, dtype=dtype, platform=platform)
    sc.build_model = build_model_b200


def uninstall():
    import sasmodels.core as sc
    if "build_model" in _ORIGINAL:
        sc.build_model = _ORIGINAL.pop("build_model")
