"""
sasmodels_b200: a B200 (sm_100a) compute engine for sasmodels plugins.

Drop-in for the polydispersity / orientation / magnetism hot path of
sasmodels (``Kernel._call_kernel`` -> ``kernel_iq.c`` -> model C):

    from sasmodels_b200 import load_model, direct_model
    model = load_model("cylinder")
    kernel = model.make_kernel([qx, qy])
    I = direct_model.call_kernel(kernel, dict(radius=20, radius_pd=0.1, ...))

or, with sasmodels installed, ``sasmodels_b200.install()`` and then
``sasmodels.core.build_model(info, platform="b200")``.
"""

from .core import build_model, install, list_models, load_model, load_model_info
from .kernel import B200Kernel, B200Model

__all__ = ["build_model", "install", "list_models", "load_model",
           "load_model_info", "B200Kernel", "B200Model"]
__version__ = "0.1.0"
