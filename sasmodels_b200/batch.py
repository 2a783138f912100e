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

import numpy as np

from . import _abi
from .core import load_model_info
from .direct_model import make_call_args

SET_FIELDS = 8
ITEM_FIELDS = 4
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
    if model == "ellipsoid":
        return max(p["radius_polar"], p["radius_equatorial"])
    if model == "core_shell_cylinder":
        return max(p["radius"] + p["thickness"], 0.5*p["length"] + p["thickness"])
    if model == "cylinder":
        return max(p["radius"], 0.5*p["length"])
    return 0.0


def rule_points(qr):
    """Gauss rule length for q*r_max (lib/adaptive.c:11290-11297)."""
    qr = np.asarray(qr)
    return np.where(qr < 10, 20, np.where(qr < 100, 76, np.where(qr < 750, 500, 5000)))


def line_call_args(info, pars, q):
    """(details, values) of one line-form set: marshaled as a 2D call at
    (q, 0); orientation dispersion is refused (the line form has no jitter
    rotation)."""
    q = np.asarray(q, 'd')
    details, values, _ = make_call_args(info, pars, [q, np.zeros_like(q)])
    kpars = info.parameters.kernel_parameters
    for d in range(details.num_active):
        p = kpars[int(details.pd_par[d])]
        if p.type == "orientation" and details.pd_length[d] > 1:
            raise ValueError("line form: %s has orientation dispersion" % p.name)
    return details, values


def _batch_fn(model):
    lib = ct.CDLL(_abi.library_path(model))
    fn = getattr(lib, "sasb200_%s_batch" % model)
    fn.argtypes = ([ct.c_int32]*4 + [ct.c_void_p]*4 + [ct.c_int32] + [ct.c_void_p]*3
                   + [ct.c_double, ct.c_int32] + [ct.c_void_p]*6)
    fn.restype = ct.c_int32
    err = getattr(lib, "sasb200_%s_last_error" % model)
    err.restype = ct.c_char_p
    return fn, err


class Population:
    """A packed population of one model on one GPU (see module doc)."""

    def __init__(self, model, sets, form="float32c", device=None, cutoff=0.0,
                 reff_mode=0, warps=8, blocks=0, items_per_warp=8, line=False):
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
        self._pack(sets)

    # ---------------------------------------------------------------- pack --
    def _pack(self, sets):
        torch = self.torch
        info = self.info
        qs, dets, vals, desc = [], [], [], []
        q_off = det_off = val_off = raw_off = iq_off = tile_off = 0
        self.nq = []
        self.num_eval = []
        self.pd_shape = []
        costs = []
        for q, pars in sets:
            q = np.ascontiguousarray(q, 'd').ravel()
            details, values = self._marshal(pars, q)
            nq, n_eval = q.size, details.num_eval
            ntile = (nq + 31)//32
            desc.append([nq, q_off, det_off, val_off, n_eval, raw_off, iq_off, tile_off])
            qs.append(q)
            dets.append(details.buffer.astype(np.int32))
            vals.append(values)
            self.nq.append(nq)
            self.num_eval.append(n_eval)
            self.pd_shape.append(tuple(details.buffer))
            q_off += nq
            det_off += details.buffer.size
            val_off += values.size
            raw_off += 2*nq + 4
            iq_off += nq
            tile_off += ntile
            rmax = 0.0 if self.line else _rmax(self.model, pars, info)
            pts = rule_points(q*rmax) if rmax > 0 else np.ones(nq)
            costs.append(pts)
        self.n_sets = len(desc)
        self.n_tiles = tile_off
        self._val_sizes = [v.size for v in vals]
        items, tile_lists = self._items(desc, costs)
        self.n_items = len(items)
        # CSR of items per (set, tile), each in mesh order
        off = np.zeros(self.n_tiles + 1, np.int32)
        flat = []
        for t in range(self.n_tiles):
            lst = sorted(tile_lists[t], key=lambda k: items[k][2])
            flat.extend(lst)
            off[t + 1] = len(flat)
        dev = dict(device=self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.d_sets = torch.as_tensor(np.array(desc, np.int32).ravel(), **dev)
            self.d_q = torch.as_tensor(np.concatenate(qs), **dev)
            self.d_det = torch.as_tensor(np.concatenate(dets), **dev)
            self.h_val = torch.as_tensor(np.concatenate(vals)).pin_memory()
            self.d_val = self.h_val.to(self.device, non_blocking=True)
            self.d_items = torch.as_tensor(np.array(items, np.int32).reshape(-1), **dev)
            self.d_tile_off = torch.as_tensor(off, **dev)
            self.d_tile_items = torch.as_tensor(np.array(flat, np.int32), **dev)
            f64 = dict(dtype=torch.float64, device=self.device)
            self.d_partials = torch.empty(max(64*self.n_items, 1), **f64)
            self.d_norms = torch.empty(4*self.n_sets, **f64)
            self.d_raw = torch.empty(raw_off, **f64)
            self.d_iq = torch.empty(iq_off, **f64)
            self.d_counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.desc = np.array(desc)
        self.stream.synchronize()

    def _marshal(self, pars, q):
        if not self.line:
            details, values, _ = make_call_args(self.info, pars, [q])
            return details, values
        return line_call_args(self.info, pars, q)

    def _items(self, desc, costs):
        """Cut every (set, tile) into mesh ranges of similar cost."""
        torch = self.torch
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        warps_resident = sms*(64 // self.warps)*self.warps // 2
        tile_cost = []
        for s, (nq, _, _, _, n_eval, _, _, tile0) in enumerate(desc):
            pts = costs[s]
            for t in range((nq + 31)//32):
                p = pts[32*t:32*t + 32]
                short = p[p <= 76]
                long_ = p[p > 76]
                per_point = (_COST_POINT + (short.max() if short.size else 0)*_COST_NODE
                             + np.sum(np.ceil(long_/32.0)*_COST_NODE + _COST_REDUCE))
                tile_cost.append((s, t, tile0 + t, n_eval, per_point))
        total = sum(n*c for _, _, _, n, c in tile_cost)
        target = max(total/(warps_resident*self.items_per_warp), 1.0)
        items, lists, cost = [], [[] for _ in range(self.n_tiles)], []
        for s, t, tile, n_eval, per_point in tile_cost:
            if n_eval == 0:
                continue
            splits = int(min(n_eval, max(1, np.ceil(n_eval*per_point/target))))
            bounds = np.linspace(0, n_eval, splits + 1).astype(int)
            for a, b in zip(bounds[:-1], bounds[1:]):
                if b > a:
                    lists[tile].append(len(items))
                    items.append((s, 32*t, int(a), int(b)))
                    cost.append((b - a)*per_point)
        order = np.argsort(-np.array(cost), kind="stable") if cost else []
        remap = np.empty(len(items), np.int64)
        remap[order] = np.arange(len(items))
        items = [items[k] for k in order]
        lists = [[int(remap[k]) for k in lst] for lst in lists]
        return items, lists

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
            self.d_val.copy_(self.h_val, non_blocking=True)
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        with self.torch.cuda.stream(self.stream):
            self.graph.replay()

    def update(self, pars_list):
        """New parameter values for the same q vectors and dispersity sizes."""
        off = 0
        host = self.h_val.numpy()
        for k, pars in enumerate(pars_list):
            details, values = self._marshal(pars, np.zeros(1))
            if tuple(details.buffer) != self.pd_shape[k]:
                raise ValueError("set %d changed its dispersity structure" % k)
            n = self._val_sizes[k]
            self.stream.synchronize()
            host[off:off + n] = values
            off += n
        if self.graph is None:
            with self.torch.cuda.stream(self.stream):
                self.d_val.copy_(self.h_val, non_blocking=True)

    # ------------------------------------------------------------- results --
    def iq(self):
        self.stream.synchronize()
        flat = self.d_iq.cpu().numpy()
        return [flat[d[6]:d[6] + d[0]] for d in self.desc]

    def raw(self):
        self.stream.synchronize()
        flat = self.d_raw.cpu().numpy()
        return [flat[d[5]:d[5] + 2*d[0] + 4] for d in self.desc]
