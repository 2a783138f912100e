"""
Marshaling of many parameter sets of one model at once.

A fit population (a bumps/DREAM generation, a surrogate's fallback points)
is many parameter sets of one model that differ in their values but share
their dispersity settings.  ``make_call_args`` marshals one set at a time
(``details.py:225-254`` via ``direct_model.py:97-154``); here the sets are
grouped by dispersity structure and each group is marshaled with array
arithmetic: one ``make_details`` per group (the loop descriptor depends only
on the mesh lengths) and the pd values and weights of all sets of the group
as rows of one matrix.  The arithmetic is the per-set arithmetic applied
elementwise (``np.linspace`` with array end points, the same exponent, one
1D sum per row for the normalisation), so every row equals what
``make_call_args`` returns for that set, bit for bit; sets the array path
does not cover (distributions other than gaussian, points clipped at a
parameter limit, vector parameters) go through ``make_call_args`` itself.
"""

import numpy as np

from .details import convert_magnetism, make_details
from .direct_model import RADIUS_MODE_ID, make_call_args
from .modelinfo import NUM_COMMON_PARS


def _fields(table, pars, active):
    """Per call parameter: (value, npts, width, nsigma, type, dispersed),
    with the defaults and the inactive rule of ``_pop_par_weights``."""
    out = []
    for p in table.call_parameters:
        value = float(pars.get(p.name, p.default))
        if p.polydisperse:
            npts = pars.get(p.name + "_pd_n", 0)
            width = pars.get(p.name + "_pd", 0.0)
            nsigma = pars.get(p.name + "_pd_nsigma", 3.0)
            dist = pars.get(p.name + "_pd_type", "gaussian")
            dispersed = not (npts == 0 or width == 0.0 or not active(p.name))
            out.append((value, int(npts), float(width), float(nsigma), dist, dispersed))
        else:
            out.append((value, 0, 0.0, 3.0, "gaussian", False))
    return out


def _allowed(table):
    names = set()
    for p in table.call_parameters:
        names.add(p.name)
        if p.polydisperse:
            names.update(p.name + s for s in ("_pd", "_pd_n", "_pd_nsigma", "_pd_type"))
    return names


def _gaussian_rows(center, width, nsigma, npts, relative, limits):
    """Vectorised GaussianDispersion.get_weights + normalisation for rows of
    (center, width); returns (x, w, ok) where ok marks rows with no point
    clipped at the limits (the others change length and go the scalar way)."""
    sigma = width*center if relative else width
    if not relative:
        center = np.zeros_like(center)
    x = center[:, None] + np.linspace(-nsigma*sigma, +nsigma*sigma, npts, axis=1)
    lb, ub = limits
    ok = np.all((x >= lb) & (x <= ub), axis=1) & (sigma != 0)
    w = np.exp((x - center[:, None])**2/(-2.0*sigma[:, None]*sigma[:, None]))
    # one 1D sum per row: a 2D reduction may add in another order
    w = w/np.array([np.sum(row) for row in w])[:, None]
    return x, w, ok


def bulk_call_args(info, pars_list, dim="1d"):
    """(details, values, is_magnetic) for every parameter dict of
    *pars_list*, as ``make_call_args(info, pars, q_vectors)`` would give
    them for a call of dimension *dim*; sets of one dispersity structure
    share one details object."""
    table = info.parameters
    npars = table.npars
    if dim == "1d":
        active = lambda name: name in table.pd_1d
    else:
        active = lambda name: name in table.pd_2d
    allowed = _allowed(table)
    vector = any(getattr(p, "length", 1) > 1 for p in table.call_parameters)
    out = [None]*len(pars_list)
    groups = {}
    q_dummy = [np.zeros(1)] if dim == "1d" else [np.zeros(1), np.zeros(1)]
    for i, pars in enumerate(pars_list):
        if RADIUS_MODE_ID not in allowed:
            pars = {k: v for k, v in pars.items() if k != RADIUS_MODE_ID}
        extra = set(pars) - allowed
        if extra:
            raise TypeError("Unused parameters in call: %s" % ", ".join(sorted(extra)))
        f = _fields(table, pars, active)
        kernel = f[NUM_COMMON_PARS:NUM_COMMON_PARS + npars]
        simple = not vector and all(d == "gaussian" and n >= 2 for _, n, _, _, d, disp
                                    in kernel if disp)
        if not simple:
            out[i] = make_call_args(info, pars, q_dummy)
            continue
        key = tuple((n, s) if disp else None for _, n, _, s, _, disp in kernel)
        groups.setdefault(key, []).append((i, pars, f))
    kpars = table.call_parameters[NUM_COMMON_PARS:NUM_COMMON_PARS + npars]
    nvalues = table.nvalues
    for key, members in groups.items():
        F = [m[2] for m in members]
        n = len(members)
        scalars = np.array([[fld[0] for fld in f] for f in F], dtype=float)
        xs, ws = [], []
        ok = np.ones(n, bool)
        for k, (p, spec) in enumerate(zip(kpars, key)):
            col = scalars[:, NUM_COMMON_PARS + k]
            if spec is None:
                # an idle orientation jitter is 0, any other idle value itself
                keep = p.relative_pd or not p.polydisperse
                xs.append((col if keep else np.zeros(n))[:, None])
                ws.append(np.ones((n, 1)))
                continue
            npts, nsigma = spec
            width = np.array([f[NUM_COMMON_PARS + k][2] for f in F])
            x, w, good = _gaussian_rows(col, width, nsigma, npts, p.relative_pd, p.limits)
            xs.append(x)
            ws.append(w)
            ok &= good
        length = np.array([x.shape[1] for x in xs])
        offset = np.cumsum(np.hstack((0, length)))
        details = make_details(info, length, offset[:-1], offset[-1])
        data_len = nvalues + 2*int(length.sum())
        pad = (32 - data_len % 32) % 32
        data = np.hstack([scalars] + xs + ws + [np.zeros((n, pad))])
        for row, (i, pars, _) in enumerate(members):
            if not ok[row]:
                out[i] = make_call_args(info, pars, q_dummy)
                continue
            values = data[row].copy()
            magnetic = convert_magnetism(table, values)
            out[i] = (details, values, magnetic)
    return out
