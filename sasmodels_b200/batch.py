"""
Whole-population evaluation: many parameter sets of one 1D model in one
persistent launch (``csrc/sas_batch.cuh``), optionally captured in a CUDA
graph so that repeated evaluations of the same population structure (the
iterations of a DREAM fit) replay without launch overhead.

    pop = Population("ellipsoid", [(q1, pars1), (q2, pars2), ...])
    pop.run()                   # enqueue on pop.stream
    curves = pop.iq()           # list of I(q) arrays (synchronises)
    pop.update([pars1b, ...])   # new values, same q and pd sizes
    pop.replay()                # graph replay

``line=True`` evaluates instead the 2D kernel along the qx axis (qy = 0) at
each set's own view angles (theta, phi), without orientation dispersion:
the line cut of an oriented 2D pattern, for models with an Iqac kernel.

The packing uses the same marshaling as a single call (``details`` and
``values`` per set, ``details.py:225-254``), concatenated.  Work items
(set, 32-q tile, mesh range) are sized by a cost model of the adaptive
quadrature (20/76/500/5000 points by q*r_max, ``lib/adaptive.c``) so that
each warp of the persistent grid gets several items of similar cost; the
items are issued longest first.
"""

import ctypes as ct
import os

import numpy as np

from . import _abi
from .core import load_model_info
from .direct_model import make_call_args

SET_FIELDS = 8
ITEM_FIELDS = 4
#: rule length up to which one lane walks a whole quadrature (sas_batch.cuh)
SHORT_RULE = 76
FORMS = {"double": 0, "float32c": 1}
LINE_FORMS = {"double": 2, "float32c": 3}

# warp-cycles per rule point in each mode, and fixed costs (arbitrary units;
# only ratios matter for splitting)
_COST_NODE = 1.0
_COST_REDUCE = 12.0
_COST_POINT = 8.0


def _rmax(model, pars, info):
    """Largest dimension at the centre of the distributions (sets the Gauss
    rule, as the model's Fq does)."""
    p = dict(info.parameters.defaults)
    p.update({k: v for k, v in pars.items() if k in p})
    return float(_rmax_arrays(model, p))


def _rmax_arrays(model, p):
    """`_rmax` of parameter values that may be arrays over sets."""
    if model == "ellipsoid":
        return np.maximum(p["radius_polar"], p["radius_equatorial"])
    if model == "core_shell_cylinder":
        return np.maximum(np.add(p["radius"], p["thickness"]),
                          np.add(0.5*np.asarray(p["length"]), p["thickness"]))
    if model == "cylinder":
        return np.maximum(p["radius"], 0.5*np.asarray(p["length"]))
    return np.zeros(())


def rule_points(qr):
    """Gauss rule length for q*r_max (lib/adaptive.c:11290-11297)."""
    qr = np.asarray(qr)
    return np.where(qr < 10, 20, np.where(qr < 100, 76, np.where(qr < 750, 500, 5000)))


def _check_line(info, details):
    kpars = info.parameters.kernel_parameters
    for d in range(details.num_active):
        p = kpars[int(details.pd_par[d])]
        if p.type == "orientation" and details.pd_length[d] > 1:
            raise ValueError("line form: %s has orientation dispersion" % p.name)


def line_call_args(info, pars, q):
    """(details, values) of one line-form set: marshaled as a 2D call at
    (q, 0); orientation dispersion is refused (the line form has no jitter
    rotation)."""
    q = np.asarray(q, 'd')
    details, values, _ = make_call_args(info, pars, [q, np.zeros_like(q)])
    _check_line(info, details)
    return details, values


def host_pack(model, info, sets, line=False, warps=8, items_per_warp=8, sms=148):
    """
    The flat arrays of a population (see csrc/sas_batch.cuh) built on the
    host: per-set marshaling through pack.bulk_call_args (bitwise the
    arrays of make_call_args), and the work items cut by the cost model.
    Returns a dict of numpy arrays and sizes.
    """
    from .pack import bulk_call_args
    qs = [np.ascontiguousarray(q, 'd').ravel() for q, _ in sets]
    args = bulk_call_args(info, [p for _, p in sets], "2d" if line else "1d")
    if line:
        for d in {id(a[0]): a[0] for a in args}.values():
            _check_line(info, d)
    n = len(sets)
    num_eval = np.array([a[0].num_eval for a in args], np.int64)
    det_all = (np.concatenate([a[0].buffer for a in args]).astype(np.int32) if n
               else np.zeros(0, np.int32))
    val_sizes = np.array([a[1].size for a in args], np.int64)
    rmax = np.array([_rmax(model, p, info) for _, p in sets]) if n else np.zeros(0)
    h = _layout(qs, num_eval, det_all, val_sizes, rmax, line, warps, items_per_warp, sms)
    h.update(pd_shape=[tuple(a[0].buffer) for a in args],
             val=np.concatenate([a[1] for a in args]) if n else np.zeros(0))
    return h


def host_pack_columns(model, info, qs, columns, line=False, warps=8, items_per_warp=8, sms=148):
    """
    The flat arrays of a population given as parameter columns (see
    pack.column_args): everything but the values, which the device packer
    expands from the returned ``columns`` table (host-marshaled values only
    for the sets the table cannot describe).
    """
    from .pack import column_args
    qs = [np.ascontiguousarray(q, 'd').ravel() for q in qs]
    n = len(qs)
    ca = column_args(info, n, columns, "2d" if line else "1d")
    if line:
        for d in {id(d): d for d in ca["details"]}.values():
            _check_line(info, d)
    p = dict(info.parameters.defaults)
    names = set(par.name for par in info.parameters.call_parameters)
    p.update({k: np.asarray(v, float) for k, v in columns.items() if k in names})
    rmax = np.broadcast_to(_rmax_arrays(model, p), (n,)).astype(float)
    h = _layout(qs, ca["num_eval"], ca["det"].ravel(), ca["val_sizes"], rmax, line, warps,
                items_per_warp, sms)
    h.update(pd_shape=[tuple(r) for r in ca["det"]], val=None, columns=ca)
    return h


def _layout(qs, num_eval, det_all, val_sizes, rmax, line, warps, items_per_warp, sms):
    """Set descriptors, concatenated q and the work items of a population."""
    n = len(qs)
    nq = np.array([q.size for q in qs], np.int64)
    det_sizes = np.full(n, det_all.size//n if n else 0, np.int64)
    ntile = (nq + 31)//32

    def offsets(sizes):
        return np.concatenate(([0], np.cumsum(sizes)[:-1])).astype(np.int64)

    desc = np.stack([nq, offsets(nq), offsets(det_sizes), offsets(val_sizes), num_eval,
                     offsets(2*nq + 4), offsets(nq), offsets(ntile)], axis=1).astype(np.int32)
    q_all = np.concatenate(qs) if n else np.zeros(0)
    # Gauss rule points per q (one node per q for the line form)
    pts = np.ones(q_all.size)
    if not line and n:
        r = np.repeat(rmax, nq)
        pts = np.where(r > 0, rule_points(r*q_all), 1.0)
    items, tile_off, tile_items = cut_items(nq, num_eval, pts, warps, items_per_warp, sms)
    return dict(nq=[int(v) for v in nq], num_eval=[int(v) for v in num_eval],
                val_sizes=list(val_sizes), desc=desc, q=q_all, det=det_all, items=items,
                tile_off=tile_off, tile_items=tile_items, n_tiles=int(ntile.sum()),
                n_items=len(items), raw_size=int((2*nq + 4).sum()), iq_size=int(nq.sum()))


def cut_items(nq, num_eval, pts, warps, items_per_warp, sms):
    """Cut every (set, 32-q tile) into mesh ranges of similar cost and order
    the items longest first.  pts: Gauss rule points of every q (all sets
    concatenated).  Returns (items int32[n, 4] = set, q0, m0, m1;
    tile_off int32[n_tiles + 1]; tile_items int32[n_items]) with each
    tile's items listed in mesh order."""
    nq = np.asarray(nq, np.int64)
    num_eval = np.asarray(num_eval, np.int64)
    ntile = (nq + 31)//32
    n_tiles = int(ntile.sum())
    warps_resident = sms*(64 // warps)*warps // 2
    if n_tiles == 0:
        return np.zeros((0, 4), np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32)
    tile_set = np.repeat(np.arange(len(nq)), ntile)
    tile_first = np.arange(n_tiles) - np.repeat(np.cumsum(ntile) - ntile, ntile)
    # q range of every tile in the concatenated q array; tiles are
    # contiguous, so reduceat over the tile starts sums exactly one tile
    q_start = np.repeat(np.cumsum(nq) - nq, ntile) + 32*tile_first
    short = np.where(pts <= SHORT_RULE, pts, 0.0)
    longc = np.where(pts > SHORT_RULE, np.ceil(pts/32.0)*_COST_NODE + _COST_REDUCE, 0.0)
    per_point = (_COST_POINT + np.maximum.reduceat(short, q_start)*_COST_NODE
                 + np.add.reduceat(longc, q_start))
    n_eval = num_eval[tile_set]
    total = float(np.sum(n_eval*per_point))
    target = max(total/(warps_resident*items_per_warp), 1.0)
    splits = np.minimum(n_eval, np.maximum(1, np.ceil(n_eval*per_point/target))).astype(np.int64)
    splits[n_eval == 0] = 0
    item_tile = np.repeat(np.arange(n_tiles), splits)
    k = np.arange(item_tile.size) - np.repeat(np.cumsum(splits) - splits, splits)
    s_t = splits[item_tile]
    n_t = n_eval[item_tile]
    m0 = (k*n_t)//s_t
    m1 = ((k + 1)*n_t)//s_t
    cost = (m1 - m0)*per_point[item_tile]
    order = np.argsort(-cost, kind="stable")
    items = np.stack([tile_set[item_tile], 32*tile_first[item_tile], m0, m1],
                     axis=1)[order].astype(np.int32)
    # positions of each tile's items (created in mesh order) after sorting
    remap = np.empty(order.size, np.int64)
    remap[order] = np.arange(order.size)
    tile_items = remap.astype(np.int32)
    tile_off = np.concatenate(([0], np.cumsum(splits))).astype(np.int32)
    return items, tile_off, tile_items


def _batch_fn(model):
    lib = ct.CDLL(_abi.library_path(model))
    fn = getattr(lib, "sasb200_%s_batch" % model)
    fn.argtypes = ([ct.c_int32]*4 + [ct.c_void_p]*4 + [ct.c_int32] + [ct.c_void_p]*3
                   + [ct.c_double, ct.c_int32] + [ct.c_void_p]*6)
    fn.restype = ct.c_int32
    err = getattr(lib, "sasb200_%s_last_error" % model)
    err.restype = ct.c_char_p
    return fn, err


def _pack_lib():
    path = os.path.join(_abi.LIB_DIR, "libsasb200_pack.so")
    if not os.path.exists(path):
        raise RuntimeError("device packer not built: %s" % path)
    lib = ct.CDLL(path)
    P, I = ct.c_void_p, ct.c_int32
    lib.sasb200_pack_values.argtypes = [I, I, I, I] + [P]*12 + [P]
    lib.sasb200_pack_values.restype = I
    lib.sasb200_pack_max_pars.restype = I
    lib.sasb200_pack_last_error.restype = ct.c_char_p
    return lib


class _Packer:
    """The per-set table of a column population in pinned host memory and on
    the device, and the launch that expands it into the values vectors
    (``sasb200_pack_values``); sets marshaled on the host are copied from
    their own pinned rows."""

    def __init__(self, ca, device, stream):
        import torch
        self.torch = torch
        self.lib = _pack_lib()
        self.stream = stream
        n, nvalues = ca["scalars"].shape
        npars = ca["npts"].shape[1]
        if npars > self.lib.sasb200_pack_max_pars():
            raise ValueError("%d kernel parameters exceed the device packer's limit" % npars)
        self.n, self.nvalues, self.npars = n, nvalues, npars
        sizes = np.asarray(ca["val_sizes"], np.int64)
        offs = np.concatenate(([0], np.cumsum(sizes)[:-1])).astype(np.int64)
        self.offs = offs
        dev_off = offs.copy()
        host_rows = sorted(ca["host_values"])
        dev_off[host_rows] = -1
        f64 = dict(dtype=torch.float64)
        self.nmag = int(ca["nmag"])
        self.h_table = torch.empty(n*(nvalues + 2*npars), **f64).pin_memory()
        self.d_table = torch.empty_like(self.h_table, device=device)
        # int32 table: npts, first, ntot, kinds (n x npars each), magnetic (n)
        self.h_itable = torch.empty(4*n*npars + n, dtype=torch.int32).pin_memory()
        self.d_itable = torch.empty_like(self.h_itable, device=device)
        self.d_flags = torch.as_tensor(ca["flags"], device=device)
        self.d_off = torch.as_tensor(dev_off, device=device)
        self.d_size = torch.as_tensor(sizes, device=device)
        self.h_rows = {r: torch.empty(int(sizes[r]), **f64).pin_memory() for r in host_rows}

    def load(self, ca):
        """Write a table (same structure) into the pinned buffers."""
        t = self.h_table.numpy()
        a = self.n*self.nvalues
        b = a + self.n*self.npars
        t[:a] = ca["scalars"].ravel()
        t[a:b] = ca["widths"].ravel()
        t[b:] = ca["nsigmas"].ravel()
        it = self.h_itable.numpy()
        m = self.n*self.npars
        for j, key in enumerate(("npts", "first", "ntot", "kinds")):
            it[j*m:(j + 1)*m] = ca[key].ravel()
        it[4*m:] = ca["magnetic"]
        for r, buf in self.h_rows.items():
            buf.numpy()[:] = ca["host_values"][r]

    def enqueue(self, d_val):
        """Copy the table to the device and expand it into d_val, on the
        stream (graph-capturable)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            self.d_table.copy_(self.h_table, non_blocking=True)
            self.d_itable.copy_(self.h_itable, non_blocking=True)
            for r, buf in self.h_rows.items():
                o = int(self.offs[r])
                d_val[o:o + buf.numel()].copy_(buf, non_blocking=True)
        a = self.n*self.nvalues
        b = a + self.n*self.npars
        base = self.d_table.data_ptr()
        ib = self.d_itable.data_ptr()
        m = 4*self.n*self.npars
        status = self.lib.sasb200_pack_values(
            self.n, self.nvalues, self.npars, self.nmag, base, base + 8*a, base + 8*b,
            ib, ib + m, ib + 2*m, ib + 3*m, self.d_flags.data_ptr(), ib + 4*m,
            self.d_off.data_ptr(), self.d_size.data_ptr(), d_val.data_ptr(),
            self.stream.cuda_stream)
        if status != 0:
            raise RuntimeError("pack_values failed (%d): %s"
                               % (status, self.lib.sasb200_pack_last_error().decode()))


class Population:
    """A packed population of one model on one GPU (see module doc)."""

    def __init__(self, model, sets, form="float32c", device=None, cutoff=0.0,
                 reff_mode=0, warps=8, blocks=0, items_per_warp=8, line=False, columns=None):
        import torch
        self.torch = torch
        self.model = model
        self.info = load_model_info(model)
        if not self.info.raw.get("f32c"):
            raise ValueError("model %s has no batched kernels" % model)
        if form not in FORMS:
            raise ValueError("form must be one of %s" % sorted(FORMS))
        self.form = form
        self.line = bool(line)
        if self.line and self.info.xy_mode != "qac":
            raise ValueError("line form needs a model with an Iqac kernel (%s is %s)"
                             % (model, self.info.xy_mode))
        self.form_code = (LINE_FORMS if self.line else FORMS)[form]
        self.cutoff = float(cutoff)
        self.reff_mode = int(reff_mode)
        self.warps = int(warps)
        self.blocks = int(blocks)
        self.items_per_warp = items_per_warp
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(self.device)
        self.fn, self.err = _batch_fn(model)
        self.graph = None
        self.columns = None
        if columns is None:
            self._pack(sets)
        else:
            self._pack_columns(sets, columns)

    @classmethod
    def from_columns(cls, model, qs, columns, **kwargs):
        """A population given as parameter columns over the q vectors `qs`:
        `columns` maps parameter names (and ``<name>_pd``, ``_pd_n``,
        ``_pd_nsigma``, ``_pd_type``) to a scalar shared by all sets or an
        array with one entry per set.  The values vectors are expanded on
        the device (``csrc/pack.cu``) from a table of a few numbers per set,
        and ``update_columns`` refreshes them the same way."""
        return cls(model, qs, columns=columns, **kwargs)

    # ---------------------------------------------------------------- pack --
    def _pack(self, sets):
        torch = self.torch
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        h = host_pack(self.model, self.info, sets, self.line, self.warps,
                      self.items_per_warp, sms)
        self._upload(h)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.h_val = torch.as_tensor(h["val"]).pin_memory()
            self.d_val = self.h_val.to(self.device, non_blocking=True)
        self.stream.synchronize()

    def _pack_columns(self, qs, columns):
        torch = self.torch
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        h = host_pack_columns(self.model, self.info, qs, columns, self.line, self.warps,
                              self.items_per_warp, sms)
        self._upload(h)
        ca = h["columns"]
        self.packer = _Packer(ca, self.device, self.stream)
        self.h_val = None
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.d_val = torch.empty(max(int(np.sum(ca["val_sizes"])), 1), dtype=torch.float64,
                                     device=self.device)
        self.packer.load(ca)
        self.packer.enqueue(self.d_val)
        self.columns = ca
        self.stream.synchronize()

    def _upload(self, h):
        torch = self.torch
        self.nq = h["nq"]
        self.num_eval = h["num_eval"]
        self.pd_shape = h["pd_shape"]
        self._val_sizes = h["val_sizes"]
        self.n_sets = len(self.nq)
        self.n_tiles = h["n_tiles"]
        self.n_items = h["n_items"]
        dev = dict(device=self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.d_sets = torch.as_tensor(h["desc"].ravel(), **dev)
            self.d_q = torch.as_tensor(h["q"], **dev)
            self.d_det = torch.as_tensor(h["det"], **dev)
            self.d_items = torch.as_tensor(h["items"].ravel(), **dev)
            self.d_tile_off = torch.as_tensor(h["tile_off"], **dev)
            self.d_tile_items = torch.as_tensor(h["tile_items"], **dev)
            f64 = dict(dtype=torch.float64, device=self.device)
            self.d_partials = torch.empty(max(64*self.n_items, 1), **f64)
            self.d_norms = torch.empty(4*self.n_sets, **f64)
            self.d_raw = torch.empty(h["raw_size"], **f64)
            self.d_iq = torch.empty(h["iq_size"], **f64)
            self.d_counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.desc = h["desc"]

    def _marshal(self, pars, q):
        if not self.line:
            details, values, _ = make_call_args(self.info, pars, [q])
            return details, values
        return line_call_args(self.info, pars, q)

    # ----------------------------------------------------------------- run --
    def run(self):
        """Enqueue one evaluation of every set on ``self.stream``."""
        torch = self.torch
        with torch.cuda.device(self.device):
            status = self.fn(self.form_code, self.warps, self.blocks, self.n_sets,
                             self.d_sets.data_ptr(), self.d_q.data_ptr(),
                             self.d_det.data_ptr(), self.d_val.data_ptr(), self.n_items,
                             self.d_items.data_ptr(), self.d_tile_off.data_ptr(),
                             self.d_tile_items.data_ptr(), self.cutoff, self.reff_mode,
                             self.d_partials.data_ptr(), self.d_norms.data_ptr(),
                             self.d_raw.data_ptr(), self.d_iq.data_ptr(),
                             self.d_counter.data_ptr(), self.stream.cuda_stream)
        if status != 0:
            raise RuntimeError("sasb200_%s_batch failed (%d): %s"
                               % (self.model, status, self.err().decode()))

    def capture(self):
        """Capture upload-of-values + evaluation in a CUDA graph."""
        torch = self.torch
        self.run()                      # first call outside capture (module load)
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.device(self.device), torch.cuda.graph(g, stream=self.stream):
            if self.columns is None:
                self.d_val.copy_(self.h_val, non_blocking=True)
            else:
                self.packer.enqueue(self.d_val)
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        with self.torch.cuda.stream(self.stream):
            self.graph.replay()

    def update_columns(self, columns):
        """New parameter columns for a population made by `from_columns`,
        with the same q vectors and dispersity sizes: the table is rewritten
        in pinned memory and expanded on the device by the next `replay()`
        (or now, on the stream, when no graph was captured)."""
        from .pack import column_args
        if self.columns is None:
            raise ValueError("update_columns needs a population made by from_columns")
        ca = column_args(self.info, self.n_sets, columns, "2d" if self.line else "1d")
        old = self.columns
        if (not np.array_equal(ca["det"], old["det"])
                or not np.array_equal(ca["val_sizes"], old["val_sizes"])
                or not np.array_equal(ca["magnetic"], old["magnetic"])
                or set(ca["host_values"]) != set(old["host_values"])):
            raise ValueError("the population changed its dispersity structure")
        self.stream.synchronize()
        self.packer.load(ca)
        self.columns = ca
        if self.graph is None:
            self.packer.enqueue(self.d_val)

    def update(self, pars_list):
        """New parameter values for the same q vectors and dispersity sizes
        (the next generation of a fit), marshaled in one pass."""
        from .pack import bulk_call_args
        if self.columns is not None:
            raise ValueError("a population made by from_columns takes update_columns")
        if len(pars_list) != self.n_sets:
            raise ValueError("expected %d parameter sets, got %d"
                             % (self.n_sets, len(pars_list)))
        args = bulk_call_args(self.info, pars_list, "2d" if self.line else "1d")
        checked = {}
        for k, (details, values, _) in enumerate(args):
            shape = checked.get(id(details))
            if shape is None:
                if self.line:
                    _check_line(self.info, details)
                shape = checked[id(details)] = tuple(details.buffer)
            if shape != self.pd_shape[k] or values.size != self._val_sizes[k]:
                raise ValueError("set %d changed its dispersity structure" % k)
        # the previous upload may still be reading the pinned buffer
        self.stream.synchronize()
        host = self.h_val.numpy()
        off = 0
        for (_, values, _), n in zip(args, self._val_sizes):
            host[off:off + n] = values
            off += n
        if self.graph is None:
            with self.torch.cuda.stream(self.stream):
                self.d_val.copy_(self.h_val, non_blocking=True)

    # ------------------------------------------------------------ fitting --
    def nllf(self, Iq, dIq, resolution=None):
        """The fit objective of every set against one data set, computed on
        the device after ``run()``/``replay()``: theory -> resolution
        smearing (a ``sasmodels_b200.resolution.Pinhole1D`` whose q_calc is
        every set's q) -> 0.5 sum(((theory - Iq)/dIq)^2)
        (``bumps_model.py:263-282``).  Returns a numpy array, one value per
        set."""
        from .resolution import nllf_sets
        nq = self.nq[0] if self.nq else 0
        if any(n != nq for n in self.nq):
            raise ValueError("nllf needs every set on the same q")
        theory = self.d_iq.view(self.n_sets, nq)
        if resolution is not None:
            if len(resolution.q_calc) != nq:
                raise ValueError("resolution q_calc has %d points, the sets %d"
                                 % (len(resolution.q_calc), nq))
            theory = resolution.apply_sets(theory, self.stream)
        out = nllf_sets(theory, Iq, dIq, self.stream)
        self.stream.synchronize()
        return out.cpu().numpy()

    # ------------------------------------------------------------- results --
    def iq(self):
        self.stream.synchronize()
        flat = self.d_iq.cpu().numpy()
        return [flat[d[6]:d[6] + d[0]] for d in self.desc]

    def raw(self):
        self.stream.synchronize()
        flat = self.d_raw.cpu().numpy()
        return [flat[d[5]:d[5] + 2*d[0] + 4] for d in self.desc]
