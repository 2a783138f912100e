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

``column_args`` prepares a population given as parameter columns for the
device packer (``csrc/pack.cu``), which expands every distribution, clipped
meshes and the magnetic conversion on the GPU.
"""

import numpy as np

from .details import convert_magnetism, make_details
from .direct_model import RADIUS_MODE_ID, make_call_args
from .modelinfo import NUM_COMMON_PARS, NUM_MAGNETIC_PARS


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


def _column(columns, name, default, n):
    """One parameter over the n sets: a scalar broadcast or an array of n."""
    v = np.asarray(columns.get(name, default))
    if v.ndim == 0:
        return np.full(n, v[()])
    if v.shape != (n,):
        raise ValueError("column %s has shape %s, expected (%d,)" % (name, v.shape, n))
    return v


#: distribution codes of the device packer (csrc/pack.cu, enum Kind)
KIND_CODES = {"gaussian": 0, "uniform": 1, "rectangle": 2, "lognormal": 3, "schulz": 4,
              "boltzmann": 5}


def _kept_ranges(kind, center, sigma, nsig, npts, limits):
    """For the sets of one parameter sharing distribution `kind` and point
    count `npts`: the linspace points of weights.dispersion (the same
    arithmetic, vectorised over rows), which of them the limits (and the
    rectangle's box) keep, and whether they form one contiguous index range.
    Returns (first, count, contiguous)."""
    from .weights import SPECS, _nodes_width
    spec = SPECS[kind]
    if spec.nodes is _nodes_width:
        x = np.linspace(center - sigma, center + sigma, npts, axis=1)
    else:
        x = center[:, None] + np.linspace(-nsig*sigma, +nsig*sigma, npts, axis=1)
    lb, ub = limits
    if spec.positive:
        lb, ub = max(lb, 1e-8), max(ub, 1e-8)
    keep = (x >= lb) & (x <= ub)
    if spec.box:
        keep &= np.fabs(x - center[:, None]) <= np.fabs(sigma)[:, None]*np.sqrt(3.0)
    count = keep.sum(axis=1)
    first = np.argmax(keep, axis=1)
    idx = np.arange(npts)[None, :]
    contiguous = np.all(keep == ((idx >= first[:, None]) & (idx < (first + count)[:, None])),
                        axis=1)
    return first, count, contiguous


def column_args(info, n_sets, columns, dim="1d"):
    """
    Marshaling of a population given as parameter columns, for the device
    packer (``csrc/pack.cu``): `columns` maps parameter names and their
    dispersity fields (``<name>_pd``, ``_pd_n``, ``_pd_nsigma``,
    ``_pd_type``) to a scalar shared by every set or an array with one entry
    per set; parameters not named keep their defaults.

    Returns a dict with the compact per-set table the device expands
    (``scalars`` [n, nvalues], ``widths``/``nsigmas`` [n, npars]; per set
    and kernel parameter ``npts`` the kept points (0 for an idle parameter),
    ``first`` the index of the first kept point among the ``ntot`` points of
    its linspace, ``kinds`` the distribution code; ``flags`` [npars];
    ``magnetic`` [n] whether the set's magnetic moments are converted), the
    ``details`` object, ``det`` buffer, ``num_eval`` and padded ``val_sizes``
    of every set, and ``host_values`` {set: values} for the sets the table
    cannot describe (a zero sigma, fewer than two points, an empty or split
    range of kept points, an "array" dispersity, a lognormal or schulz
    jitter centred on zero), which ``make_call_args`` marshals.  Every
    distribution of the plugin API and the magnetic conversion run on the
    device; a device-packed set's values equal ``make_call_args``'s points
    bit for bit, its weights and magnetic components to an ulp or two
    (exp, log, lgamma, sin, cos).
    """
    table = info.parameters
    npars = table.npars
    n = int(n_sets)
    if any(getattr(p, "length", 1) > 1 for p in table.call_parameters):
        raise ValueError("%s has vector parameters: marshal it set by set" % info.id)
    allowed = _allowed(table)
    columns = {k: v for k, v in columns.items()
               if not (k == RADIUS_MODE_ID and RADIUS_MODE_ID not in allowed)}
    extra = set(columns) - allowed
    if extra:
        raise TypeError("Unused parameters in call: %s" % ", ".join(sorted(extra)))
    active = table.pd_1d if dim == "1d" else table.pd_2d
    call = table.call_parameters
    scalars = np.empty((n, table.nvalues))
    for j, p in enumerate(call):
        scalars[:, j] = _column(columns, p.name, p.default, n).astype(float)
    kpars = call[NUM_COMMON_PARS:NUM_COMMON_PARS + npars]
    widths = np.zeros((n, npars))
    nsigmas = np.full((n, npars), 3.0)
    npts = np.zeros((n, npars), np.int32)
    first = np.zeros((n, npars), np.int32)
    ntot = np.zeros((n, npars), np.int32)
    kinds = np.zeros((n, npars), np.int32)
    lengths = np.ones((n, npars), np.int64)
    flags = np.array([(1 if p.relative_pd else 0) | (2 if (p.relative_pd or not p.polydisperse)
                                                     else 0) for p in kpars], np.int32)
    host = np.zeros(n, bool)
    for k, p in enumerate(kpars):
        if not p.polydisperse:
            continue
        nn = _column(columns, p.name + "_pd_n", 0, n).astype(np.int64)
        w = _column(columns, p.name + "_pd", 0.0, n).astype(float)
        ns = _column(columns, p.name + "_pd_nsigma", 3.0, n).astype(float)
        kind = _column(columns, p.name + "_pd_type", "gaussian", n)
        dispersed = (nn != 0) & (w != 0.0) & (p.name in active)
        value = scalars[:, NUM_COMMON_PARS + k]
        sigma = w*value if p.relative_pd else w
        center = value if p.relative_pd else np.zeros(n)
        code = np.array([KIND_CODES.get(str(t), -1) for t in kind], np.int32)
        ok = dispersed & (code >= 0) & (nn >= 2) & (sigma != 0)
        # a zero linspace step takes numpy's other formula, for every row of
        # a vectorised call: such sets go the scalar way
        ok &= (code == KIND_CODES["uniform"]) | (ns != 0)
        if not p.relative_pd:
            ok &= (code != KIND_CODES["lognormal"]) & (code != KIND_CODES["schulz"])
        cnt = np.zeros(n, np.int64)
        fst = np.zeros(n, np.int64)
        for name, c in KIND_CODES.items():
            for m in np.unique(nn[ok & (code == c)]):
                rows = np.nonzero(ok & (code == c) & (nn == m))[0]
                f0, c0, contiguous = _kept_ranges(name, center[rows], sigma[rows],
                                                  ns[rows], int(m), p.limits)
                fst[rows], cnt[rows] = f0, c0
                ok[rows] &= contiguous & (c0 > 0)
        host |= dispersed & ~ok
        npts[:, k] = np.where(ok, cnt, 0)
        first[:, k] = np.where(ok, fst, 0)
        ntot[:, k] = np.where(ok, nn, 0)
        kinds[:, k] = np.where(ok, code, 0)
        widths[:, k] = np.where(ok, w, 0.0)
        nsigmas[:, k] = ns
        lengths[:, k] = np.where(ok, cnt, 1)
    magnetic = np.zeros(n, np.int32)
    if table.nmagnetic:
        mag = scalars[:, table.nvalues - NUM_MAGNETIC_PARS*table.nmagnetic:]
        magnetic[:] = np.any(mag[:, ::NUM_MAGNETIC_PARS] != 0.0, axis=1)
    det_len = 4*table.max_pd + 4
    det = np.empty((n, det_len), np.int32)
    num_eval = np.empty(n, np.int64)
    val_sizes = np.empty(n, np.int64)
    details = [None]*n
    host_values = {}
    dev = np.nonzero(~host)[0]
    if dev.size:
        shapes, inverse = np.unique(lengths[dev], axis=0, return_inverse=True)
        inverse = inverse.ravel()
        for g, length in enumerate(shapes):
            offset = np.cumsum(np.hstack((0, length)))
            d = make_details(info, length, offset[:-1], offset[-1])
            rows = dev[inverse == g]
            data_len = table.nvalues + 2*int(length.sum())
            det[rows] = d.buffer
            num_eval[rows] = d.num_eval
            val_sizes[rows] = data_len + (32 - data_len % 32) % 32
            for r in rows:
                details[r] = d
    q_dummy = [np.zeros(1)] if dim == "1d" else [np.zeros(1), np.zeros(1)]
    for r in np.nonzero(host)[0]:
        pars = {}
        for k, v in columns.items():
            v = np.asarray(v)
            v = v[()] if v.ndim == 0 else v[r]
            pars[k] = v.item() if hasattr(v, "item") else v
        d, values, _ = make_call_args(info, pars, q_dummy)
        det[r] = d.buffer
        num_eval[r] = d.num_eval
        val_sizes[r] = values.size
        details[r] = d
        host_values[int(r)] = values
    return dict(scalars=scalars, widths=widths, nsigmas=nsigmas, npts=npts, first=first,
                ntot=ntot, kinds=kinds, flags=flags, magnetic=magnetic, nmag=table.nmagnetic,
                lengths=lengths, details=details, det=det, num_eval=num_eval,
                val_sizes=val_sizes, host_values=host_values)


def columns_from_sets(info, pars_list):
    """Parameter columns of a list of parameter dicts (for column_args):
    every name any set gives, with the parameter's default where a set
    leaves it out."""
    defaults = info.parameters.defaults
    names = sorted(set().union(*[set(p) for p in pars_list])) if pars_list else []
    cols = {}
    for k in names:
        if k in defaults:
            fill = defaults[k]
        elif k.endswith("_pd_type"):
            fill = "gaussian"
        else:
            fill = 3.0 if k.endswith("_pd_nsigma") else 0.0
        vals = [p.get(k, fill) for p in pars_list]
        cols[k] = (np.array(vals, dtype=object) if k.endswith("_pd_type")
                   else np.array(vals, dtype=float))
    return cols
