"""
Host-side model metadata for the B200 backend.

The B200 kernels are built per model.  Each build writes a JSON sidecar next
to the shared library that records the model's parameter table exactly as the
sasmodels plugin API defines it (``sasmodels/modelinfo.py``: ``Parameter``
at 283-378, ``ParameterTable`` at 399-672, ``ModelInfo`` at 1018-1228).  At
run time this module rebuilds the subset of those objects the call path reads
(``details.make_kernel_args``, ``direct_model.get_mesh``, ``Kernel.Fq``), so
that a machine without the sasmodels package can still drive the kernels.

When sasmodels is importable, :func:`from_sasmodels` adapts a live
``sasmodels.modelinfo.ModelInfo`` into the same JSON form, which is what the
build step does.
"""

import json
import math
import os

import numpy as np

#: Maximum number of simultaneously polydisperse parameters
#: (``sasmodels/modelinfo.py:38``).
MAX_PD = 5
#: scale and background lead every values vector (``modelinfo.py:48-53``).
NUM_COMMON_PARS = 2
#: up_frac_i, up_frac_f, up_theta, up_phi (``modelinfo.py:55``).
NUM_MAGFIELD_PARS = 4
#: M0, mtheta, mphi per sld parameter (``modelinfo.py:56``).
NUM_MAGNETIC_PARS = 3

_INF = float("inf")


def _num(x):
    """JSON-safe float (inf is spelled as a string)."""
    if isinstance(x, (int, float)) and math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return x


def _unnum(x):
    if x == "inf":
        return _INF
    if x == "-inf":
        return -_INF
    return x


class Parameter:
    """
    One call parameter.  The fields mirror ``sasmodels.modelinfo.Parameter``
    (``modelinfo.py:283-378``) for the attributes the call path uses.
    """
    def __init__(self, name, units="", default=0.0, limits=(-_INF, _INF),
                 ptype="", description="", polydisperse=False,
                 relative_pd=False, length=1):
        self.id = self.name = name
        self.units = units
        self.default = default
        self.limits = tuple(limits)
        self.type = ptype
        self.description = description
        self.polydisperse = polydisperse
        self.relative_pd = relative_pd
        self.length = length

    def as_dict(self):
        return dict(name=self.name, units=self.units, default=_num(self.default),
                    limits=[_num(v) for v in self.limits], type=self.type,
                    description=self.description,
                    polydisperse=bool(self.polydisperse),
                    relative_pd=bool(self.relative_pd), length=int(self.length))

    @classmethod
    def from_dict(cls, d):
        return cls(d["name"], d.get("units", ""), _unnum(d["default"]),
                   [_unnum(v) for v in d["limits"]], d["type"],
                   d.get("description", ""), d["polydisperse"],
                   d["relative_pd"], d.get("length", 1))

    def __repr__(self):
        return "P<%s>" % self.name


class ParameterTable:
    """
    The parameter bookkeeping needed to lay out the ``values`` vector and the
    ``CallDetails`` buffer (``modelinfo.py:446-506``).

    *call_parameters* is the full list: scale, background, the kernel
    parameters (vectors expanded), then the magnetic block when the model has
    sld parameters (``modelinfo.py:634-672``).
    """
    def __init__(self, call_parameters, kernel_parameters, npars, nmagnetic,
                 theta_offset, max_pd, is_asymmetric):
        self.call_parameters = call_parameters
        self.kernel_parameters = kernel_parameters
        self.npars = npars
        self.nmagnetic = nmagnetic
        self.nvalues = NUM_COMMON_PARS + npars
        if nmagnetic:
            self.nvalues += NUM_MAGFIELD_PARS + NUM_MAGNETIC_PARS*nmagnetic
        self.theta_offset = theta_offset
        self.max_pd = max_pd
        self.is_asymmetric = is_asymmetric
        self.common_parameters = call_parameters[:NUM_COMMON_PARS]
        self.iq_parameters = [p for p in kernel_parameters
                              if p.type not in ('orientation', 'magnetic')]
        self.orientation_parameters = [p for p in kernel_parameters
                                       if p.type == 'orientation']
        self.form_volume_parameters = [p for p in kernel_parameters
                                       if p.type == 'volume']
        self.has_2d = any(p.type in ('orientation', 'magnetic')
                          for p in kernel_parameters)
        # modelinfo.py:497-500
        self.pd_1d = set(p.name for p in call_parameters
                         if p.polydisperse and p.type not in ('orientation', 'magnetic'))
        self.pd_2d = set(p.name for p in call_parameters if p.polydisperse)
        self.defaults = {p.id: p.default for p in call_parameters}

    def __getitem__(self, key):
        for par in self.call_parameters:
            if par.name == key:
                return par
        raise KeyError("unknown parameter %r" % key)

    def __contains__(self, key):
        return any(par.name == key for par in self.call_parameters)

    @property
    def sld_indices(self):
        """Indices into the kernel parameter vector of the sld parameters,
        in call order.  These are the slds replaced by their effective
        magnetic values (``generate.py:1125``: ``MAGNETIC_PARS``)."""
        return [k - NUM_COMMON_PARS for k, p in enumerate(self.call_parameters)
                if p.type == 'sld']


class ModelInfo:
    """
    Per-model metadata read by the call path (subset of
    ``sasmodels.modelinfo.ModelInfo``, ``modelinfo.py:1018-1228``), plus the
    fields the B200 build derived from the model's C sources (``xy_mode``,
    ``have_shell``).
    """
    def __init__(self, d):
        self.id = d["id"]
        self.name = d["name"]
        self.have_Fq = bool(d["have_Fq"])
        self.radius_effective_modes = d.get("radius_effective_modes") or []
        self.xy_mode = d["xy_mode"]
        self.have_shell = bool(d["have_shell"])
        self.single = bool(d.get("single", True))
        self.structure_factor = bool(d.get("structure_factor", False))
        self.tests = d.get("tests", [])
        kernel = [Parameter.from_dict(p) for p in d["kernel_parameters"]]
        call = [Parameter.from_dict(p) for p in d["call_parameters"]]
        self.parameters = ParameterTable(
            call, kernel, d["npars"], d["nmagnetic"], d["theta_offset"],
            d["max_pd"], d["is_asymmetric"])
        self.raw = d

    def as_dict(self):
        return self.raw

    def __repr__(self):
        return "ModelInfo(%s)" % self.id


def from_sasmodels(info, xy_mode, have_shell):
    """
    Convert a live ``sasmodels.modelinfo.ModelInfo`` into the JSON dict the
    B200 build stores beside each model library.
    """
    table = info.parameters
    d = dict(
        id=info.id, name=info.name, have_Fq=bool(info.have_Fq),
        radius_effective_modes=list(info.radius_effective_modes or []),
        xy_mode=xy_mode, have_shell=bool(have_shell),
        single=bool(getattr(info, 'single', True)),
        structure_factor=bool(getattr(info, 'structure_factor', False)),
        npars=int(table.npars), nmagnetic=int(table.nmagnetic),
        nvalues=int(table.nvalues), theta_offset=int(table.theta_offset),
        max_pd=int(table.max_pd), is_asymmetric=bool(table.is_asymmetric),
        kernel_parameters=[_par_dict(p) for p in table.kernel_parameters],
        call_parameters=[_par_dict(p) for p in table.call_parameters],
    )
    return d


def _par_dict(p):
    return Parameter(p.name, p.units, p.default, p.limits, p.type,
                     p.description, bool(p.polydisperse),
                     bool(p.relative_pd), int(p.length or 1)).as_dict()


def load_info_json(path):
    with open(path) as fid:
        return ModelInfo(json.load(fid))


def as_b200_info(info):
    """Accept either our :class:`ModelInfo` or a sasmodels ModelInfo."""
    if isinstance(info, ModelInfo):
        return info
    from . import generate
    return generate.info_from_sasmodels(info)


def expand_defaults(info, pars=None):
    """Parameter dict with defaults filled in (``modelinfo.py:202-257``
    restricted to scalar parameters)."""
    result = dict(info.parameters.defaults)
    if pars:
        result.update(pars)
    return result


def default_q(n=3):
    return np.array([0.01, 0.1, 0.2][:n])
