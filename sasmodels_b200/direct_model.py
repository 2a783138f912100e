"""
Parameter dict -> dispersity mesh -> kernel call, for callers that run
without the sasmodels package (with it installed, ``install()`` lets the
reference's own ``sasmodels.direct_model`` drive the B200 kernels).

The mesh must be the one the reference builds for the same dict
(``sasmodels/direct_model.py:41-154``): one (value, points, weights) entry
per call parameter, in the table's order; a parameter is polydisperse only
if it may be (``polydisperse``), is active for the kernel's dimension
(``pd_1d``/``pd_2d``) and has both points and a width; an idle orientation
parameter contributes a single point at zero jitter (its value is the view
angle, the jitter is the distribution); unknown names are an error.
"""

from . import weights
from .details import make_kernel_args

#: parameter name that selects the effective-radius mode in call_Fq
#: (``sasmodels/product.py:143``).
RADIUS_MODE_ID = "radius_effective_mode"

#: dispersity entries of a parameter `p`: p_pd, p_pd_n, p_pd_nsigma, p_pd_type
_PD_SUFFIXES = ("_pd", "_pd_n", "_pd_nsigma", "_pd_type")


def call_kernel(calculator, pars, cutoff=0., mono=False):
    """I(q) of *calculator* (a kernel from ``make_kernel``) for the
    parameter dict *pars*."""
    call_details, values, magnetic = _marshal(calculator, pars, mono)
    return calculator(call_details, values, cutoff, magnetic)


def call_Fq(calculator, pars, cutoff=0., mono=False):
    """(<F>, <F^2>, R_eff, V_shell, V_form/V_shell) for *pars*; the entry
    ``radius_effective_mode`` of *pars* selects the effective radius
    (default 1)."""
    pars = dict(pars)
    mode = int(pars.pop(RADIUS_MODE_ID, 1.0))
    call_details, values, magnetic = _marshal(calculator, pars, mono)
    return calculator.Fq(call_details, values, cutoff, magnetic, mode)


def _marshal(calculator, pars, mono):
    mesh = get_mesh(calculator.info, pars, dim=calculator.dim, mono=mono)
    return make_kernel_args(calculator, mesh)


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
    """[(value, points, weights)] for every call parameter of *model_info*,
    from the dict *values*; *dim* ('1d', '2d', or anything else for all
    polydisperse parameters) picks which dispersities are active, *mono*
    switches them all off."""
    table = model_info.parameters
    known = set()
    for p in table.call_parameters:
        known.add(p.name)
        if p.polydisperse:
            known.update(p.name + sfx for sfx in _PD_SUFFIXES)
    unused = [k for k in values if k not in known]
    if unused:
        raise TypeError("Unused parameters in call: %s" % ", ".join(unused))
    if mono:
        active = ()
    elif dim == '1d':
        active = table.pd_1d
    elif dim == '2d':
        active = table.pd_2d
    else:
        active = None          # every polydisperse parameter
    return [_parameter_mesh(p, values, active is None or p.name in active)
            for p in table.call_parameters]


def _parameter_mesh(p, values, active):
    """(value, points, weights) of call parameter *p* from its entries in
    *values* (defaults: the table's value, no points, width 0, 3 sigmas,
    gaussian)."""
    value = float(values.get(p.name, p.default))
    if not p.polydisperse:
        return value, [value], [1.0]
    npts = values.get(p.name + "_pd_n", 0)
    width = values.get(p.name + "_pd", 0.0)
    if not active or npts == 0 or width == 0.0:
        # idle: the value itself, or for orientation jitter no jitter
        return value, [value if p.relative_pd else 0.0], [1.0]
    points, wts = weights.get_weights(values.get(p.name + "_pd_type", "gaussian"), npts,
                                      width, values.get(p.name + "_pd_nsigma", 3.0), value,
                                      p.limits, p.relative_pd)
    return value, points, wts
