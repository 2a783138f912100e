"""
Learned surrogate for the polydisperse cylinder: log I(q | R, L, R_pd, L_pd,
contrast, q, orientation flag), with the plain kernels as its data source,
its judge and its fallback.

* The network (``csrc/mlp.cu``) is 7 inputs (padded to 16) -> 4 x 256 SiLU
  -> 1, BF16 weights and activations, FP32 accumulation on the tcgen05
  tensor cores, trained here with the project's own forward, backward,
  weight-gradient and Adam kernels.
* Training data: parameter sets drawn uniformly / log-uniformly over the
  domain below, evaluated by the plain engines: flag 1 = the 1D orientation
  average (``cylinder`` Fq, batched engine), flag 0 = the oriented 2D kernel
  at theta = 90, phi = 0 without jitter, with q along qx.
* The intensity is exactly quadratic in the contrast, so the network learns
  y = log I at unit contrast and ``2 log|contrast|`` is added back.
* Predicted error: a calibration table of the held-out |error| (99th
  percentile) over (log q, log L, log R) bins.  Points whose predicted error
  exceeds the tolerance (default 1 % in log I), or that fall outside the
  training domain, are recomputed by the plain kernel.

Domain: R in [10, 300] A, L in [20, 3000] A, R_pd and L_pd in [0, 0.3]
(gaussian, 35 points, 3 sigma when > 0), contrast in [-5, 5], q in
[1e-3, 0.5] 1/A.
"""

import ctypes as ct
import math
import os

import numpy as np

from ._abi import LIB_DIR

HID = 256
NIN = 16
TM = 128
DOMAIN = dict(radius=(10.0, 300.0), length=(20.0, 3000.0), rpd=(0.0, 0.3),
              lpd=(0.0, 0.3), contrast=(-5.0, 5.0), q=(1e-3, 0.5))
PD_N = 35


def _lib():
    path = os.path.join(LIB_DIR, "libsasb200_mlp.so")
    if not os.path.exists(path):
        raise RuntimeError("surrogate library not built: %s" % path)
    lib = ct.CDLL(path)
    P, I, F = ct.c_void_p, ct.c_int32, ct.c_float
    lib.sasb200_mlp_forward.argtypes = [I, I, P, P, P, P, P, P, P, P, P, P]
    lib.sasb200_mlp_backward.argtypes = [I, I, P, P, P, P, P, P, P]
    lib.sasb200_gemm_nt.argtypes = [I, I, I, I, I, P, P, I, P, P, P]
    lib.sasb200_transpose_bf16.argtypes = [I, I, P, P, P]
    lib.sasb200_row_dot.argtypes = [I, I, P, P, P, P]
    lib.sasb200_mse_grad.argtypes = [I, I, P, P, P, P, P]
    lib.sasb200_adam.argtypes = [I, I, P, P, P, P, F, F, F, F, I, P, P, I, I, P]
    lib.sasb200_mlp_features.argtypes = [I, I, P, P, P, P, P, P, P, P, P]
    for name in ("sasb200_mlp_forward", "sasb200_mlp_backward", "sasb200_gemm_nt",
                 "sasb200_transpose_bf16", "sasb200_row_dot", "sasb200_mse_grad",
                 "sasb200_adam", "sasb200_mlp_features"):
        getattr(lib, name).restype = I
    lib.sasb200_mlp_last_error.restype = ct.c_char_p
    return lib


def pad128(n):
    return ((n + TM - 1)//TM)*TM


class MLP:
    """Weights, optimiser state and the device kernels of the surrogate."""

    def __init__(self, device=None, seed=0):
        import torch
        self.torch = torch
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.lib = _lib()
        self.stream = torch.cuda.Stream(self.device)
        rng = np.random.default_rng(seed)
        shapes = [(HID, NIN), (HID, HID), (HID, HID), (HID, HID)]
        f32 = dict(dtype=torch.float32, device=self.device)
        self.W, self.b = [], []
        for l, (o, i) in enumerate(shapes):
            fan_in = 7 if l == 0 else i
            bound = math.sqrt(6.0/fan_in)
            w = rng.uniform(-bound, bound, (o, i))
            if l == 0:
                w[:, 7:] = 0.0
            self.W.append(torch.as_tensor(w, **f32))
            self.b.append(torch.zeros(o, **f32))
        self.w_out = torch.as_tensor(rng.uniform(-1, 1, HID)/math.sqrt(HID), **f32)
        self.b_out = torch.zeros(1, **f32)
        self.params = self.W + self.b + [self.w_out, self.b_out]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._sync_bf16()
        self._scratch_n = 0

    # bf16 copies used by the kernels
    def _sync_bf16(self):
        torch = self.torch
        self.Wb = [w.to(torch.bfloat16).contiguous() for w in self.W]
        self.WTb = [w.t().contiguous().to(torch.bfloat16) for w in self.W]

    def _ptrs(self, tensors):
        arr = (ct.c_void_p*len(tensors))(*[t.data_ptr() for t in tensors])
        return arr

    def _check(self, status, what):
        if status != 0:
            raise RuntimeError("%s failed (%d): %s" % (what, status,
                                                      self.lib.sasb200_mlp_last_error().decode()))

    def _scratch(self, n_pad):
        torch = self.torch
        if n_pad <= self._scratch_n:
            return
        bf = dict(dtype=torch.bfloat16, device=self.device)
        f32 = dict(dtype=torch.float32, device=self.device)
        self.z_save = torch.empty(4*n_pad*HID, **bf)
        self.h_save = torch.empty(4*n_pad*HID, **bf)
        self.dz_save = torch.empty(4*n_pad*HID, **bf)
        self.t_a = torch.empty(HID*n_pad, **bf)        # transposed dZ
        self.t_b = torch.empty(HID*n_pad, **bf)        # transposed h / x
        self.out = torch.empty(n_pad, **f32)
        self.dout = torch.empty(n_pad, **f32)
        self.sq = torch.empty(n_pad, **f32)
        self.splits = 8
        self.gW = [torch.empty(self.splits*HID*(NIN if l == 0 else HID), **f32)
                   for l in range(4)]
        self.gb = [torch.empty(HID, **f32) for _ in range(4)]
        self.gw = torch.empty(HID, **f32)
        self.gbo = torch.empty(1, **f32)
        self._scratch_n = n_pad

    # ----------------------------------------------------------- kernels --
    def forward(self, x, n, save=False):
        """out[n_pad] for features x (bf16 [n_pad x 16]), on self.stream."""
        n_pad = x.shape[0]
        self._scratch(n_pad)
        st = self.stream.cuda_stream
        w = self._ptrs(self.Wb)
        b = self._ptrs(self.b)
        self._check(self.lib.sasb200_mlp_forward(
            n, n_pad, x.data_ptr(), w, b, self.w_out.data_ptr(), self.b_out.data_ptr(),
            self.out.data_ptr(), self.z_save.data_ptr() if save else None,
            self.h_save.data_ptr() if save else None, self.err.data_ptr(), st), "mlp_forward")
        return self.out[:n_pad]

    def gradients(self, x, y, n):
        """Loss and gradients of one batch, all on self.stream: returns
        (loss, dW split partials [4], db [4], dw_out, db_out)."""
        torch = self.torch
        n_pad = x.shape[0]
        self._scratch(n_pad)
        st = self.stream.cuda_stream
        lib = self.lib
        self._check(lib.sasb200_mlp_forward(
            n, n_pad, x.data_ptr(), self._ptrs(self.Wb), self._ptrs(self.b),
            self.w_out.data_ptr(), self.b_out.data_ptr(), self.out.data_ptr(),
            self.z_save.data_ptr(), self.h_save.data_ptr(), self.err.data_ptr(), st), "forward")
        self._check(lib.sasb200_mse_grad(n, n_pad, self.out.data_ptr(), y.data_ptr(),
                                         self.dout.data_ptr(), self.sq.data_ptr(), st), "mse")
        self._check(lib.sasb200_mlp_backward(n, n_pad, self._ptrs(self.WTb), self.w_out.data_ptr(),
                                             self.dout.data_ptr(), self.z_save.data_ptr(),
                                             self.dz_save.data_ptr(), self.err.data_ptr(), st),
                    "backward")
        plane = n_pad*HID
        for l in range(4):
            nb = NIN if l == 0 else HID
            dz = self.dz_save[l*plane:(l + 1)*plane]
            self._check(lib.sasb200_transpose_bf16(n_pad, HID, dz.data_ptr(),
                                                   self.t_a.data_ptr(), st), "transpose")
            if l == 0:
                src, cols = x, NIN
            else:
                src, cols = self.h_save[(l - 1)*plane:l*plane], HID
            self._check(lib.sasb200_transpose_bf16(n_pad, cols, src.data_ptr(),
                                                   self.t_b.data_ptr(), st), "transpose")
            self._check(lib.sasb200_gemm_nt(HID, nb, n_pad, n_pad, n_pad, self.t_a.data_ptr(),
                                            self.t_b.data_ptr(), self.splits,
                                            self.gW[l].data_ptr(), self.err.data_ptr(), st),
                        "gemm_nt")
            self._check(lib.sasb200_row_dot(HID, n_pad, self.t_a.data_ptr(), None,
                                            self.gb[l].data_ptr(), st), "row_dot")
        h3 = self.h_save[3*plane:4*plane]
        self._check(lib.sasb200_transpose_bf16(n_pad, HID, h3.data_ptr(), self.t_b.data_ptr(), st),
                    "transpose")
        self._check(lib.sasb200_row_dot(HID, n_pad, self.t_b.data_ptr(), self.dout.data_ptr(),
                                        self.gw.data_ptr(), st), "row_dot")
        with torch.cuda.stream(self.stream):
            self.gbo.copy_(self.dout[:n_pad].sum().reshape(1))
            loss = self.sq[:n].mean()
        return loss, self.gW, self.gb, self.gw, self.gbo

    def train_step(self, x, y, n, lr, b1=0.9, b2=0.999, eps=1e-8):
        loss, dW, db, gw, gbo = self.gradients(x, y, n)
        self.step_count += 1
        st = self.stream.cuda_stream
        lib = self.lib
        for l in range(4):
            nb = NIN if l == 0 else HID
            self._check(lib.sasb200_adam(HID*nb, self.splits, dW[l].data_ptr(), self.W[l].data_ptr(),
                                         self.m[l].data_ptr(), self.v[l].data_ptr(), lr, b1, b2, eps,
                                         self.step_count, self.Wb[l].data_ptr(),
                                         self.WTb[l].data_ptr(), HID, nb, st), "adam")
        for k, g in enumerate(db + [gw, gbo]):
            p = self.params[4 + k]
            self._check(lib.sasb200_adam(p.numel(), 1, g.data_ptr(), p.data_ptr(),
                                         self.m[4 + k].data_ptr(), self.v[4 + k].data_ptr(), lr,
                                         b1, b2, eps, self.step_count, None, None, 0, 0, st),
                        "adam")
        return loss

    def features(self, radius, length, rpd, lpd, contrast, q, flag):
        """bf16 [n_pad x 16] features on the device from float64 arrays."""
        torch = self.torch
        n = len(q)
        n_pad = pad128(n)
        arrs = [torch.as_tensor(np.ascontiguousarray(a, 'd'), device=self.device)
                for a in (radius, length, rpd, lpd, contrast, q, flag)]
        x = torch.empty((n_pad, NIN), dtype=torch.bfloat16, device=self.device)
        with torch.cuda.stream(self.stream):
            self._check(self.lib.sasb200_mlp_features(n, n_pad, *[a.data_ptr() for a in arrs],
                                                      x.data_ptr(), self.stream.cuda_stream),
                        "features")
        return x, n

    def errors(self):
        return int(self.err.item())

    def state(self):
        return {k: [t.detach().cpu().numpy() for t in v] if isinstance(v, list)
                else v.detach().cpu().numpy()
                for k, v in (("W", self.W), ("b", self.b), ("w_out", self.w_out),
                             ("b_out", self.b_out))}

    def load_state(self, st):
        torch = self.torch
        for l in range(4):
            self.W[l].copy_(torch.as_tensor(st["W"][l]))
            self.b[l].copy_(torch.as_tensor(st["b"][l]))
        self.w_out.copy_(torch.as_tensor(st["w_out"]))
        self.b_out.copy_(torch.as_tensor(st["b_out"]).reshape(1))
        self._sync_bf16()
