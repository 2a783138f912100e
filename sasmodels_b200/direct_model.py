"""
Parameter dict -> dispersity mesh -> kernel call.

Same call path as ``sasmodels/direct_model.py:41-154``: a caller that used
``sasmodels.direct_model.call_kernel(kernel, pars)`` with a DLL kernel gets
the same mesh, the same packed arrays and so the same integral from a
:class:`sasmodels_b200.kernel.B200Kernel`.
"""

from . import weights
from .details import make_kernel_args

#: parameter name that selects the effective-radius mode in call_Fq
#: (``sasmodels/product.py:143``).
RADIUS_MODE_ID = "radius_effective_mode"


def call_kernel(calculator, pars, cutoff=0., mono=False):
    """I(q) for *pars* (``direct_model.py:41-59``)."""
    mesh = get_mesh(calculator.info, pars, dim=calculator.dim, mono=mono)
    call_details, values, is_magnetic = make_kernel_args(calculator, mesh)
    return calculator(call_details, values, cutoff, is_magnetic)


def call_Fq(calculator, pars, cutoff=0., mono=False):
    """(F1, F2, R_eff, V_shell, V_form/V_shell) for *pars*
    (``direct_model.py:61-77``)."""
    pars = dict(pars)
    R_eff_type = int(pars.pop(RADIUS_MODE_ID, 1.0))
    mesh = get_mesh(calculator.info, pars, dim=calculator.dim, mono=mono)
    call_details, values, is_magnetic = make_kernel_args(calculator, mesh)
    return calculator.Fq(call_details, values, cutoff, is_magnetic, R_eff_type)


class _CallShape:
    """The attributes of a Kernel that make_kernel_args reads."""
    def __init__(self, info, dim):
        import numpy as np
        self.info = info
        self.dim = dim
        self.dtype = np.dtype('d')


def make_call_args(model_info, pars, q_vectors, mono=False):
    """(call_details, values, is_magnetic) for *pars* at *q_vectors* without
    building a kernel: the arrays a kernel call (or a batch) consumes."""
    dim = '2d' if len(q_vectors) == 2 else '1d'
    pars = dict(pars)
    if RADIUS_MODE_ID not in model_info.parameters:
        # a call argument of Fq, except for P@S where it is a parameter
        pars.pop(RADIUS_MODE_ID, None)
    mesh = get_mesh(model_info, pars, dim=dim, mono=mono)
    return make_kernel_args(_CallShape(model_info, dim), mesh)


def get_mesh(model_info, values, dim='1d', mono=False):
    """
    One (value, dispersity, weights) tuple per call parameter; parameters not
    active for *dim* are monodisperse (``direct_model.py:97-124``).
    """
    parameters = model_info.parameters
    if mono:
        active = lambda name: False
    elif dim == '1d':
        active = lambda name: name in parameters.pd_1d
    elif dim == '2d':
        active = lambda name: name in parameters.pd_2d
    else:
        active = lambda name: True
    values = dict(values)
    mesh = [_pop_par_weights(p, values, active(p.name))
            for p in parameters.call_parameters]
    if values:
        raise TypeError(f"Unused parameters in call: {', '.join(values.keys())}")
    return mesh


def _pop_par_weights(parameter, values, active=True):
    """
    Distribution for one parameter from name, name_pd, name_pd_n,
    name_pd_nsigma and name_pd_type, defaulting to n=0, nsigma=3, gaussian
    (``direct_model.py:127-154``).
    """
    value = float(values.pop(parameter.name, parameter.default))
    if parameter.polydisperse:
        npts = values.pop(parameter.name+'_pd_n', 0)
        width = values.pop(parameter.name+'_pd', 0.0)
        nsigma = values.pop(parameter.name+'_pd_nsigma', 3.0)
        distribution = values.pop(parameter.name+'_pd_type', 'gaussian')
        relative = parameter.relative_pd
        if npts == 0 or width == 0.0 or not active:
            # Orientation parameters carry the view angle as the value and the
            # jitter in the distribution, so an idle jitter is 0, not the angle.
            pd = [value if relative else 0.0], [1.0]
        else:
            pd = weights.get_weights(distribution, npts, width, nsigma,
                                     value, parameter.limits, relative)
    else:
        pd = [value], [1.0]
    return value, pd[0], pd[1]
