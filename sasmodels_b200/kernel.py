"""
The B200 implementation of the sasmodels compute-engine interface.

:class:`B200Model` / :class:`B200Kernel` follow ``sasmodels/kernel.py``
(``KernelModel`` 13-32, ``Kernel`` 35-205): ``make_kernel(q_vectors)``
returns a kernel whose ``__call__``/``Iq``/``Fq`` take
``(call_details, values, cutoff, magnetic[, radius_effective_mode])`` and
whose ``result`` array has the DLL layout (``kerneldll.py:445-447``):
``nout*nq`` F^2 (and F) slots then total weight, weighted form volume,
weighted shell volume and weighted effective radius.

Device memory is owned by torch.  q is uploaded once per kernel; each call
stages ``details`` and ``values`` through pinned host buffers on the
kernel's own CUDA stream, launches the sm_100a driver through the C-ABI and
reads the result back.  :meth:`B200Kernel.Fq_device` keeps everything on
the device for callers that chain further GPU work.

A kernel instance is not thread-safe (it owns one result buffer, as the DLL
kernel does); a model may be shared between threads.
"""

import ctypes as ct

import numpy as np

from . import _abi
from .details import validate_call

try:  # be an instance of the reference's engine classes when available
    from sasmodels.kernel import Kernel as _KernelBase
    from sasmodels.kernel import KernelModel as _KernelModelBase
except Exception:  # sasmodels not installed: same interface, no base class
    _KernelBase = object
    _KernelModelBase = object


def _torch():
    import torch
    return torch


def _require_cuda(device):
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError("B200 backend needs a CUDA device; none is visible")
    dev = torch.device(device if device is not None else "cuda")
    if dev.type != "cuda":
        raise RuntimeError("B200 backend runs on CUDA devices only, got %s" % dev)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def locality_order(qx, qy, bits=10):
    """
    Permutation that walks the (qx, qy) points along a Morton (Z-order) curve
    of the plane, so the 32 points a warp takes are close together.  Nearby
    points see nearby |q|, q_ab and q_c for every orientation, so the lanes of
    a warp follow the same branches of the model (J1 series vs asymptotic,
    adaptive quadrature order) instead of diverging.
    """
    def quantise(v):
        lo, hi = float(v.min()), float(v.max())
        scale = (2**bits - 1)/(hi - lo) if hi > lo else 0.0
        return np.rint((v - lo)*scale).astype(np.uint64)
    ix, iy = quantise(qx), quantise(qy)
    code = np.zeros(len(qx), np.uint64)
    for b in range(bits):
        code |= ((ix >> np.uint64(b)) & np.uint64(1)) << np.uint64(2*b)
        code |= ((iy >> np.uint64(b)) & np.uint64(1)) << np.uint64(2*b + 1)
    return np.argsort(code, kind="stable")


def locality_order_device(qx, qy, bits=10):
    """:func:`locality_order` computed where the tensors live (same
    quantisation, round-half-even, bit interleave and stable sort, so the
    same permutation); returns an int64 tensor on their device."""
    torch = _torch()

    def quantise(v):
        lo, hi = v.min(), v.max()
        span = hi - lo
        scale = torch.where(span > 0, (2**bits - 1)/span, torch.zeros_like(span))
        return torch.round((v - lo)*scale).to(torch.int64)
    ix, iy = quantise(qx), quantise(qy)
    code = torch.zeros_like(ix)
    for b in range(bits):
        code |= ((ix >> b) & 1) << (2*b)
        code |= ((iy >> b) & 1) << (2*b + 1)
    return torch.argsort(code, stable=True)


class QInput:
    """q points for one kernel: 1D ``q`` or interleaved ``(qx, qy)`` pairs,
    uploaded once (``kernelcuda.py:386-422`` does the same per make_kernel).
    2D points are uploaded in caller order and permuted on the device into
    :func:`locality_order` (``order_dev[i]`` is the caller's index of device
    slot i); results are put back in caller order on the device."""

    def __init__(self, q_vectors, device, reorder=True):
        torch = _torch()
        q_vectors = [np.ascontiguousarray(v, 'd').ravel() for v in q_vectors]
        self.q_vectors = q_vectors
        self.nq = int(q_vectors[0].size)
        self.is_2d = len(q_vectors) == 2
        self.order_dev = None
        self._order = None
        if self.is_2d:
            qx, qy = q_vectors
            q = np.empty(2*self.nq, 'd')
            q[0::2] = qx
            q[1::2] = qy
        elif len(q_vectors) == 1:
            q = q_vectors[0]
        else:
            raise ValueError("q_vectors must be [q] or [qx, qy]")
        self.dtype = np.dtype('d')
        if not self.nq:
            self.q_dev = torch.zeros(2, dtype=torch.float64, device=device)
            return
        q_dev = torch.as_tensor(q, device=device)
        if self.is_2d and reorder and self.nq > 32:
            pairs = q_dev.view(self.nq, 2)
            self.order_dev = locality_order_device(pairs[:, 0], pairs[:, 1])
            q_dev = pairs.index_select(0, self.order_dev).reshape(-1)
        self.q_dev = q_dev

    @property
    def order(self):
        """Host copy of ``order_dev`` (None when the points keep their
        order)."""
        if self._order is None and self.order_dev is not None:
            self._order = self.order_dev.cpu().numpy()
        return self._order

    def release(self):
        self.q_dev = None


FP64_NAMES = (None, "double", "d", "float64", np.float64, "double!")
FP32C_NAMES = ("float32c",)
#: the reference's single-precision names: this backend has no plain FP32
#: build of the plugin C (generate.convert_type), so these run the
#: FP32-compensated form, which is more accurate than it, with a warning
SINGLE_NAMES = ("single", "float", "f", "float32", np.float32, "single!", "fast")


class B200Model(_KernelModelBase):
    """
    Compute engine for one model on one CUDA device.

    *dtype* selects the form: ``"double"`` runs the model plugin's own C in
    FP64; ``"float32c"`` runs the hand-written FP32-compensated physics where
    the model has it: FP32 bulk arithmetic, FP64 phases and FP64 sums.
    The reference's single-precision names (``"single"``, ``"float32"``,
    ``"fast"``) also select the FP32-compensated form and say so with a
    ``UserWarning``: it is not the reference's plain FP32 arithmetic
    (``generate.convert_type``), it is within 1e-5 of FP64.  Models without
    FP32c physics run the FP64 form for either.  Results are always float64
    arrays.

    *model_info* is the caller's model description (ours, or a sasmodels
    ``ModelInfo`` when the model was built through the reference's
    ``core.build_model``); it is exposed unchanged as ``info``, so callers
    read their own objects back.  *meta* is this backend's description of
    the same model (parameter table and library metadata) used internally;
    it defaults to *model_info*.
    """
    def __init__(self, model_info, dtype="double", device=None, lib_dir=None, meta=None):
        self.info = model_info
        self.meta = meta if meta is not None else model_info
        if dtype in FP64_NAMES:
            form = "double"
        elif dtype in FP32C_NAMES or dtype in SINGLE_NAMES:
            form = "float32c" if self.meta.raw.get("f32c") else "double"
            if dtype in SINGLE_NAMES:
                import warnings
                what = ("the FP32-compensated form (FP32 amplitudes with FP64 phases "
                        "and sums, within 1e-5 of FP64)" if form == "float32c"
                        else "the FP64 form (no FP32 physics for this model)")
                warnings.warn("sasmodels_b200: dtype %r runs %s for %s, not the plain "
                              "single-precision build of the reference"
                              % (dtype, what, self.meta.id), UserWarning, stacklevel=2)
        else:
            raise ValueError("unsupported dtype %r" % (dtype,))
        self.form = form
        self.dtype = np.dtype('d')
        self.device = device
        self.lib = _abi.load_library(self.meta.id, lib_dir, form)

    def make_kernel(self, q_vectors, reorder=True):
        return B200Kernel(self, q_vectors, reorder=reorder)

    def release(self):
        pass


class B200Kernel(_KernelBase):
    """Callable kernel bound to one set of q points."""

    def __init__(self, model, q_vectors, device=None, reorder=True):
        torch = _torch()
        self.model = model
        self.info = model.info
        self.meta = model.meta
        self.dtype = model.dtype
        self.device = _require_cuda(device if device is not None else model.device)
        self.stream = torch.cuda.Stream(self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.q_input = QInput(q_vectors, self.device, reorder)
            self.dim = '2d' if self.q_input.is_2d else '1d'
            nq = self.q_input.nq
            nout = 2 if self.meta.have_Fq else 1
            self.result = np.empty(nq*nout + 4, 'd')
            self._result_dev = torch.zeros(nq*nout + 4, dtype=torch.float64,
                                           device=self.device)
            self._result_pin = torch.empty(nq*nout + 4, dtype=torch.float64,
                                           pin_memory=True)
        self._ws = None
        self._result_caller = None
        self._pin_values = None
        self._pin_details = None
        self._dev_values = None
        self._dev_details = None
        #: tile code handed to the C-ABI (0 = the autotuner's cached choice
        #: for this call shape, else the library's)
        self.tile = 0
        self._tuning = False
        self.lib = model.lib

    # ------------------------------------------------------------ staging --
    def _grow(self, attr, n, dtype, pinned):
        torch = _torch()
        buf = getattr(self, attr)
        if buf is None or buf.numel() < n:
            size = max(n, 64)
            if pinned:
                buf = torch.empty(size, dtype=dtype, pin_memory=True)
            else:
                buf = torch.empty(size, dtype=dtype, device=self.device)
            setattr(self, attr, buf)
        return buf

    def upload(self, call_details, values):
        """Stage details/values on the kernel stream; returns device tensors."""
        torch = _torch()
        details = np.ascontiguousarray(call_details.buffer, np.int32)
        values = np.ascontiguousarray(values, 'd')
        validate_call(self.meta, details, values)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            pin_d = self._grow("_pin_details", details.size, torch.int32, True)
            pin_v = self._grow("_pin_values", values.size, torch.float64, True)
            # the previous call's copies must be done before reuse
            self.stream.synchronize()
            pin_d[:details.size].numpy()[:] = details
            pin_v[:values.size].numpy()[:] = values
            dev_d = self._grow("_dev_details", details.size, torch.int32, False)
            dev_v = self._grow("_dev_values", values.size, torch.float64, False)
            dev_d[:details.size].copy_(pin_d[:details.size], non_blocking=True)
            dev_v[:values.size].copy_(pin_v[:values.size], non_blocking=True)
        return dev_d, dev_v

    def workspace(self, variant, n_mesh, tile=None):
        torch = _torch()
        tile = self.tile if tile is None else tile
        need = self.lib.workspace_bytes(variant, self.q_input.nq, n_mesh, tile)
        if self._ws is None or self._ws.numel() < need:
            with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
                self._ws = torch.empty(max(need, 256), dtype=torch.uint8,
                                       device=self.device)
        return self._ws

    # ------------------------------------------------------------- launch --
    def variant(self, magnetic):
        if self.dim == '1d':
            return "Iq"
        return "Imagnetic" if magnetic else "Iqxy"

    def launch(self, variant, details_dev, values_dev, pd_start, pd_stop,
               cutoff, radius_effective_mode, result_dev=None, tile=None):
        """Enqueue one driver call on ``self.stream``; all arrays on device."""
        result_dev = self._result_dev if result_dev is None else result_dev
        if tile is None and self.tile == 0 and not self._tuning:
            # a tile the autotuner measured for this call shape, if any
            from .autotune import cached_tile
            tile = cached_tile(self, variant, pd_stop - pd_start)
        tile = int(self.tile if tile is None else tile)
        ws = self.workspace(variant, pd_stop - pd_start, tile)
        self.lib.call(variant, self.q_input.nq, int(pd_start), int(pd_stop),
                      details_dev.data_ptr(), values_dev.data_ptr(),
                      self.q_input.q_dev.data_ptr(), result_dev.data_ptr(),
                      float(cutoff), int(radius_effective_mode),
                      ws.data_ptr(), ws.numel(), tile,
                      self.stream.cuda_stream)
        return result_dev

    def _call_kernel(self, call_details, values, cutoff, magnetic,
                     radius_effective_mode):
        torch = _torch()
        dev_d, dev_v = self.upload(call_details, values)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.launch(self.variant(magnetic), dev_d, dev_v, 0,
                        call_details.num_eval, cutoff, radius_effective_mode)
            res = self._result_dev
            order = self.q_input.order_dev
            if order is not None:
                # slot i holds the caller's point order[i]
                nq = self.q_input.nq
                if self._result_caller is None:
                    self._result_caller = torch.empty_like(res)
                self._result_caller[nq:] = res[nq:]
                self._result_caller[:nq].index_copy_(0, order, res[:nq])
                res = self._result_caller
            self._result_pin[:res.numel()].copy_(res, non_blocking=True)
        self.stream.synchronize()
        self.result[:] = self._result_pin.numpy()

    # ------------------------------------------- reference engine interface --
    def Iq(self, call_details, values, cutoff, magnetic):
        """scale/V_shell * <F^2> + background (``kernel.py:80-99``)."""
        _, F2, _, shell_volume, _ = self.Fq(call_details, values, cutoff,
                                            magnetic, radius_effective_mode=0)
        combined_scale = values[0]/shell_volume
        background = values[1]
        return combined_scale*F2 + background
    __call__ = Iq

    def Fq(self, call_details, values, cutoff, magnetic, radius_effective_mode=0):
        """(<F>, <F^2>, R_eff, V_shell, V_form/V_shell) normalised by the
        total weight (``kernel.py:101-188``)."""
        self._call_kernel(call_details, values, cutoff, magnetic,
                          radius_effective_mode)
        nq = self.q_input.nq
        nout = 2 if self.meta.have_Fq and self.dim == '1d' else 1
        total_weight = self.result[nout*nq + 0]
        if total_weight == 0.:
            total_weight = 1.
        form_volume = self.result[nout*nq + 1]/total_weight
        shell_volume = self.result[nout*nq + 2]/total_weight
        radius_effective = self.result[nout*nq + 3]/total_weight
        if shell_volume == 0.:
            shell_volume = 1.
        F1 = self.result[1:nout*nq:nout]/total_weight if nout == 2 else None
        F2 = self.result[0:nout*nq:nout]/total_weight
        return F1, F2, radius_effective, shell_volume, form_volume/shell_volume

    # ------------------------------------------------------ device results --
    def Iq_device(self, details_dev, values_dev, num_eval, scale, background,
                  cutoff=0., magnetic=False, out=None):
        """
        I(q) left on the device: the driver call plus the FP64 normalisation
        scale/V_shell*F^2/sum(w) + background, all enqueued on the kernel
        stream.  Returns a float64 tensor of length nq.
        """
        torch = _torch()
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            res = self.launch(self.variant(magnetic), details_dev, values_dev,
                              0, num_eval, cutoff, 0)
            nq = self.q_input.nq
            nout = 2 if self.meta.have_Fq and self.dim == '1d' else 1
            tail = res[nout*nq:nout*nq + 4]
            total = torch.where(tail[0] == 0, torch.ones_like(tail[0]), tail[0])
            shell = tail[2]/total
            shell = torch.where(shell == 0, torch.ones_like(shell), shell)
            F2 = res[0:nout*nq:nout]/total
            I = (scale/shell)*F2 + background
            if self.q_input.order_dev is not None:
                I = torch.empty_like(I).index_copy_(0, self.q_input.order_dev, I)
            if out is not None:
                out.copy_(I)
                return out
            return I

    def release(self):
        self._ws = None
        self._result_caller = None
        if self.q_input is not None:
            self.q_input.release()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
