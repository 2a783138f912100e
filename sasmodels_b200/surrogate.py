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
* Predicted error: a second network of the same shape (the error gate,
  same kernels) trained on fresh sets to predict the local envelope of the
  first network's |log I error|, with per-tolerance thresholds calibrated
  on held-out sets judged by the plain FP64 kernel (at most 0.05 % of the
  accepted calibration points off by more than the tolerance).  Points
  whose predicted error exceeds the tolerance (default 1 % in log I), or
  that fall outside the training domain, are recomputed by the plain
  kernel.

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
#: linear learning-rate warm-up of the training schedule, in steps
WARMUP_STEPS = 200


def _lib():
    path = os.path.join(LIB_DIR, "libsasb200_mlp.so")
    if not os.path.exists(path):
        raise RuntimeError("surrogate library not built: %s" % path)
    lib = ct.CDLL(path)
    P, I, F = ct.c_void_p, ct.c_int32, ct.c_float
    lib.sasb200_mlp_forward.argtypes = [I, I, P, P, P, P, P, P, P, P, P, P, P]
    lib.sasb200_mlp_backward.argtypes = [I, I, P, P, P, P, P, P, P]
    lib.sasb200_gemm_nt.argtypes = [I, I, I, I, I, P, P, I, P, P, P]
    lib.sasb200_transpose_bf16.argtypes = [I, I, P, P, P]
    lib.sasb200_loss_grad.argtypes = [I, I, P, P, F, P, P, P]
    lib.sasb200_adam.argtypes = [I, I, P, P, P, P, F, F, F, F, I, P, P, I, I, P]
    lib.sasb200_lr_schedule.argtypes = [P, P, I, I, F, F, F, P]
    lib.sasb200_adam_multi.argtypes = [I, P, P, P, P, P, P, P, P, P, P, P, F, F, F, P]
    lib.sasb200_col_sums.argtypes = [I, I, P, P, P, P, P]
    lib.sasb200_col_sum_parts.argtypes = [I]
    lib.sasb200_mlp_features.argtypes = [I, I, P, P, P, P, P, P, P, P, P, P]
    lib.sasb200_mlp_pack.argtypes = [P, P, P, P, P, P]
    lib.sasb200_mlp_infer.argtypes = [I, I, P, P, P, P, P, P, P, P, P, P, I, P]
    lib.sasb200_mlp_serve.argtypes = [I, I, P, P, P, P, P, P, P, P, P, P, I, P]
    lib.sasb200_mlp_pack_t.argtypes = [P, P, P, P, P]
    lib.sasb200_mlp_backward_p.argtypes = [I, I, P, P, P, P, P, P, I, P]
    for name in ("sasb200_mlp_forward", "sasb200_mlp_backward", "sasb200_gemm_nt",
                 "sasb200_transpose_bf16", "sasb200_loss_grad",
                 "sasb200_adam", "sasb200_mlp_features", "sasb200_mlp_pack",
                 "sasb200_mlp_infer", "sasb200_mlp_serve", "sasb200_mlp_image_bytes",
                 "sasb200_mlp_pack_t", "sasb200_mlp_image_t_bytes", "sasb200_mlp_backward_p",
                 "sasb200_lr_schedule", "sasb200_adam_multi",
                 "sasb200_col_sums", "sasb200_col_sum_parts"):
        getattr(lib, name).restype = I
    lib.sasb200_mlp_last_error.restype = ct.c_char_p
    return lib


def pad128(n):
    return ((n + TM - 1)//TM)*TM


class MLP:
    """Weights, optimiser state and the device kernels of the surrogate."""

    def __init__(self, device=None, seed=0, stream=None):
        import torch
        self.torch = torch
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.lib = _lib()
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        self._side = [torch.cuda.Stream(self.device) for _ in range(4)]
        rng = np.random.default_rng(seed)
        shapes = [(HID, NIN), (HID, HID), (HID, HID), (HID, HID)]
        f32 = dict(dtype=torch.float32, device=self.device)
        self.W, self.b = [], []
        for l, (o, i) in enumerate(shapes):
            fan_in = 15 if l == 0 else i
            bound = math.sqrt(6.0/fan_in)
            w = rng.uniform(-bound, bound, (o, i))
            if l == 0:
                w[:, 15:] = 0.0
            self.W.append(torch.as_tensor(w, **f32))
            self.b.append(torch.zeros(o, **f32))
        self.w_out = torch.as_tensor(rng.uniform(-1, 1, HID)/math.sqrt(HID), **f32)
        self.b_out = torch.zeros(1, **f32)
        self.params = self.W + self.b + [self.w_out, self.b_out]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step_count = 0
        #: Huber threshold of the training loss (<= 0: squared error)
        self.huber = 0.0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.img = torch.empty(self.lib.sasb200_mlp_image_bytes(), dtype=torch.uint8,
                               device=self.device)
        self.img_t = torch.empty(self.lib.sasb200_mlp_image_t_bytes(), dtype=torch.uint8,
                                 device=self.device)
        self._packed = None
        self._infer_out = None
        self._sync_bf16()
        self._scratch_n = 0

    # bf16 copies used by the kernels
    def _sync_bf16(self):
        torch = self.torch
        self._wversion = getattr(self, "_wversion", 0) + 1
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
        # per layer (the four weight-gradient chains run concurrently):
        # transposed dZ, transposed h / x, column-sum partials
        self.t_a = [torch.empty(HID*n_pad, **bf) for _ in range(4)]
        self.t_b = [torch.empty(HID*n_pad, **bf) for _ in range(4)]
        self.out = torch.empty(n_pad, **f32)
        self.dout = torch.empty(n_pad, **f32)
        self.sq = torch.empty(n_pad, **f32)
        parts = self.lib.sasb200_col_sum_parts(n_pad)*HID
        self.cs_part = [torch.empty(parts, **f32) for _ in range(5)]
        self.splits = 32     # split-K of the weight gradients: 64+ CTAs at batch 8192
        self.gW = [torch.empty(self.splits*HID*(NIN if l == 0 else HID), **f32)
                   for l in range(4)]
        self.gb = [torch.empty(HID, **f32) for _ in range(4)]
        self.gw = torch.empty(HID, **f32)
        self.gbo = torch.empty(1, **f32)
        self._scratch_n = n_pad

    # ----------------------------------------------------------- kernels --
    def _pack(self):
        """Refresh the chunked weight image of the inference kernel after the
        bf16 weights changed (training steps, loads)."""
        key = (self.step_count, self._wversion)
        if self._packed == key:
            return
        self._pack_kernels()
        self._packed = key

    def _pack_kernels(self):
        self._check(self.lib.sasb200_mlp_pack(*[w.data_ptr() for w in self.Wb],
                                              self.img.data_ptr(), self.stream.cuda_stream),
                    "mlp_pack")
        self._check(self.lib.sasb200_mlp_pack_t(*[w.data_ptr() for w in self.WTb[1:]],
                                                self.img_t.data_ptr(), self.stream.cuda_stream),
                    "mlp_pack_t")

    def infer(self, x, x_lo, n, blocks=0):
        """Inference only: out[n_pad] for features x + x_lo through the
        persistent pipelined kernel (mlp_infer), on self.stream."""
        torch = self.torch
        n_pad = x.shape[0]
        if self._infer_out is None or self._infer_out.numel() < n_pad:
            self._infer_out = torch.empty(n_pad, dtype=torch.float32, device=self.device)
        self._pack()
        self._check(self.lib.sasb200_mlp_infer(
            n, n_pad, x.data_ptr(), x_lo.data_ptr(), self.img.data_ptr(), self._ptrs(self.b),
            self.w_out.data_ptr(), self.b_out.data_ptr(), self._infer_out.data_ptr(), None, None,
            self.err.data_ptr(), int(blocks), self.stream.cuda_stream), "mlp_infer")
        return self._infer_out[:n_pad]

    def serve(self, x, x_lo, n, blocks=0):
        """Inference only, through the overlapped kernel (mlp_serve): the
        hidden activations of :meth:`infer` with the output dot summed in
        another order; on self.stream."""
        torch = self.torch
        n_pad = x.shape[0]
        if self._infer_out is None or self._infer_out.numel() < n_pad:
            self._infer_out = torch.empty(n_pad, dtype=torch.float32, device=self.device)
        self._pack()
        self._check(self.lib.sasb200_mlp_serve(
            n, n_pad, x.data_ptr(), x_lo.data_ptr(), self.img.data_ptr(), self._ptrs(self.b),
            self.w_out.data_ptr(), self.b_out.data_ptr(), self._infer_out.data_ptr(), None, None,
            self.err.data_ptr(), int(blocks), self.stream.cuda_stream), "mlp_serve")
        return self._infer_out[:n_pad]

    def forward(self, x, x_lo, n, save=False):
        """out[n_pad] for features x + x_lo (bf16 [n_pad x 16] each), on
        self.stream."""
        n_pad = x.shape[0]
        self._scratch(n_pad)
        st = self.stream.cuda_stream
        w = self._ptrs(self.Wb)
        b = self._ptrs(self.b)
        self._check(self.lib.sasb200_mlp_forward(
            n, n_pad, x.data_ptr(), x_lo.data_ptr(), w, b, self.w_out.data_ptr(),
            self.b_out.data_ptr(),
            self.out.data_ptr(), self.z_save.data_ptr() if save else None,
            self.h_save.data_ptr() if save else None, self.err.data_ptr(), st), "mlp_forward")
        return self.out[:n_pad]

    def gradients(self, x, x_lo, y, n):
        """Loss and gradients of one batch, all on self.stream: returns
        (loss, dW split partials [4], db [4], dw_out, db_out)."""
        self._scratch(x.shape[0])
        self._pack()
        return self._gradient_kernels(x, x_lo, y, n)

    def _gradient_kernels(self, x, x_lo, y, n):
        torch = self.torch
        n_pad = x.shape[0]
        st = self.stream.cuda_stream
        lib = self.lib
        # forward with the z/h planes through the overlapped kernel, backward
        # through the pipelined persistent kernel (weights streamed from the
        # packed images)
        self._check(lib.sasb200_mlp_serve(
            n, n_pad, x.data_ptr(), x_lo.data_ptr(), self.img.data_ptr(), self._ptrs(self.b),
            self.w_out.data_ptr(), self.b_out.data_ptr(), self.out.data_ptr(),
            self.z_save.data_ptr(), self.h_save.data_ptr(), self.err.data_ptr(), 0, st),
            "forward")
        self._check(lib.sasb200_loss_grad(n, n_pad, self.out.data_ptr(), y.data_ptr(),
                                          float(self.huber), self.dout.data_ptr(),
                                          self.sq.data_ptr(), st), "loss")
        self._check(lib.sasb200_mlp_backward_p(n, n_pad, self.img_t.data_ptr(),
                                               self.w_out.data_ptr(), self.dout.data_ptr(),
                                               self.z_save.data_ptr(), self.dz_save.data_ptr(),
                                               self.err.data_ptr(), 0, st), "backward")
        # the weight-gradient chain of each layer (transposes, split-K GEMM,
        # bias column sums) depends only on the planes: the four chains run on
        # side streams forked from self.stream and joined before it goes on,
        # so together they fill the SMs that one chain leaves idle
        plane = n_pad*HID
        fork = torch.cuda.Event()
        fork.record(self.stream)
        joins = []
        for l in range(4):
            side = self._side[l]
            side.wait_event(fork)
            ss = side.cuda_stream
            nb = NIN if l == 0 else HID
            dz = self.dz_save[l*plane:(l + 1)*plane]
            t_a, t_b = self.t_a[l], self.t_b[l]
            self._check(lib.sasb200_transpose_bf16(n_pad, HID, dz.data_ptr(), t_a.data_ptr(), ss),
                        "transpose")
            if l == 0:
                src, cols = x, NIN
            else:
                src, cols = self.h_save[(l - 1)*plane:l*plane], HID
            self._check(lib.sasb200_transpose_bf16(n_pad, cols, src.data_ptr(), t_b.data_ptr(), ss),
                        "transpose")
            self._check(lib.sasb200_gemm_nt(HID, nb, n_pad, n_pad, n_pad, t_a.data_ptr(),
                                            t_b.data_ptr(), self.splits,
                                            self.gW[l].data_ptr(), self.err.data_ptr(), ss),
                        "gemm_nt")
            # bias gradient: column sums of the dZ plane (zero on padding rows)
            self._check(lib.sasb200_col_sums(n_pad, HID, dz.data_ptr(), None,
                                             self.cs_part[l].data_ptr(), self.gb[l].data_ptr(), ss),
                        "col_sums")
            done = torch.cuda.Event()
            done.record(side)
            joins.append(done)
        # output weights: columns of the last h plane weighted by dout
        h3 = self.h_save[3*plane:4*plane]
        self._check(lib.sasb200_col_sums(n_pad, HID, h3.data_ptr(), self.dout.data_ptr(),
                                         self.cs_part[4].data_ptr(), self.gw.data_ptr(), st),
                    "col_sums")
        for done in joins:
            self.stream.wait_event(done)
        with torch.cuda.stream(self.stream):
            self.gbo.copy_(self.dout[:n_pad].sum().reshape(1))
            loss = self.sq[:n].mean()
        return loss, self.gW, self.gb, self.gw, self.gbo

    def train_step(self, x, x_lo, y, n, lr, b1=0.9, b2=0.999, eps=1e-8, reduce=None):
        """One Adam step on one batch; returns the loss (a device scalar).

        `reduce`, when given, makes this a data-parallel step: it is called
        on self.stream with the list from `reduced_gradients` and must
        average it in place over the replicas (``multigpu.allreduce_mean``:
        one all-reduce of one flat bucket), after which every replica
        applies the same update."""
        if reduce is None:
            loss, dW, db, gw, gbo = self.gradients(x, x_lo, y, n)
            self.apply_gradients(dW + db + [gw, gbo], lr, self.splits, b1, b2, eps)
            return loss
        grads = self.reduced_gradients(x, x_lo, y, n)
        with self.torch.cuda.stream(self.stream):
            reduce(grads)
        self.apply_gradients(grads[1:], lr, 1, b1, b2, eps)
        return grads[0][0]

    def reduced_gradients(self, x, x_lo, y, n):
        """[loss (1 element), dW_1..dW_4, db_1..db_4, dw_out, db_out] of one
        batch as fp32 device tensors, the weight gradients summed over their
        split-K partials: the ≈200k numbers a data-parallel step exchanges."""
        loss, dW, db, gw, gbo = self.gradients(x, x_lo, y, n)
        with self.torch.cuda.stream(self.stream):
            dW = [g.view(self.splits, -1).sum(0) for g in dW]
            return [loss.reshape(1).clone()] + dW + [g.clone() for g in db + [gw, gbo]]

    def capture_training(self, x_all, x_lo_all, y_all, batch, lr, total, step0, warmup=200,
                         b1=0.9, b2=0.999, eps=1e-8):
        """:class:`TrainingGraph` of one whole training step on `batch` rows
        of (x_all, x_lo_all, y_all) chosen by an index buffer, with the
        learning rate schedule of :meth:`Surrogate._train` (lr, total steps,
        linear warm-up over `warmup` steps, cosine decay) advancing on the
        device from schedule step `step0`."""
        return TrainingGraph(self, x_all, x_lo_all, y_all, batch, lr, total, step0, warmup,
                             b1, b2, eps)

    def apply_gradients(self, grads, lr, splits, b1=0.9, b2=0.999, eps=1e-8):
        """Adam update from [dW_1..dW_4 (each `splits` partials), db_1..db_4,
        dw_out, db_out], refreshing the bf16 weight copies; on self.stream."""
        dW, rest = grads[:4], grads[4:]
        self.step_count += 1
        st = self.stream.cuda_stream
        lib = self.lib
        for l in range(4):
            nb = NIN if l == 0 else HID
            self._check(lib.sasb200_adam(HID*nb, splits, dW[l].data_ptr(), self.W[l].data_ptr(),
                                         self.m[l].data_ptr(), self.v[l].data_ptr(), lr, b1, b2, eps,
                                         self.step_count, self.Wb[l].data_ptr(),
                                         self.WTb[l].data_ptr(), HID, nb, st), "adam")
        for k, g in enumerate(rest):
            p = self.params[4 + k]
            self._check(lib.sasb200_adam(p.numel(), 1, g.data_ptr(), p.data_ptr(),
                                         self.m[4 + k].data_ptr(), self.v[4 + k].data_ptr(), lr,
                                         b1, b2, eps, self.step_count, None, None, 0, 0, st),
                        "adam")

    def features(self, radius, length, rpd, lpd, contrast, q, flag):
        """Compensated bf16 features (hi, lo) [n_pad x 16] on the device from
        float64 arrays (host arrays, or device tensors already on this
        network's stream)."""
        torch = self.torch
        n = len(q)
        n_pad = pad128(n)
        arrs = [a.contiguous() if isinstance(a, torch.Tensor) else
                torch.as_tensor(np.ascontiguousarray(a, 'd'), device=self.device)
                for a in (radius, length, rpd, lpd, contrast, q, flag)]
        x = torch.empty((n_pad, NIN), dtype=torch.bfloat16, device=self.device)
        x_lo = torch.empty((n_pad, NIN), dtype=torch.bfloat16, device=self.device)
        with torch.cuda.stream(self.stream):
            self._check(self.lib.sasb200_mlp_features(n, n_pad, *[a.data_ptr() for a in arrs],
                                                      x.data_ptr(), x_lo.data_ptr(),
                                                      self.stream.cuda_stream),
                        "features")
        return x, x_lo, n

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


# --------------------------------------------------------------------------
# data, training, calibration and inference with fallback
# --------------------------------------------------------------------------

def sample_sets(n_sets, rng, flag=None, low_pd_frac=0.0, low_pd_max=0.08):
    """Parameter sets drawn over the training domain (log-uniform sizes,
    uniform polydispersities and contrast, random orientation flag).  With
    low_pd_frac > 0 that fraction of the sets draws its dispersities from
    [0, low_pd_max] instead, oversampling the sharply oscillating curves the
    network finds hardest."""
    lo, hi = DOMAIN["radius"]
    R = np.exp(rng.uniform(np.log(lo), np.log(hi), n_sets))
    lo, hi = DOMAIN["length"]
    L = np.exp(rng.uniform(np.log(lo), np.log(hi), n_sets))
    rpd = rng.uniform(*DOMAIN["rpd"], n_sets)
    lpd = rng.uniform(*DOMAIN["lpd"], n_sets)
    if low_pd_frac > 0:
        low = rng.uniform(0, 1, n_sets) < low_pd_frac
        rpd[low] = rng.uniform(0, low_pd_max, low.sum())
        lpd[low] = rng.uniform(0, low_pd_max, low.sum())
    contrast = rng.uniform(*DOMAIN["contrast"], n_sets)
    f = rng.integers(0, 2, n_sets) if flag is None else np.full(n_sets, flag)
    return dict(radius=R, length=L, rpd=rpd, lpd=lpd, contrast=contrast, flag=f)


def sample_q(nq, rng):
    lo, hi = DOMAIN["q"]
    return np.sort(np.exp(rng.uniform(np.log(lo), np.log(hi), nq)))


def model_pars(R, L, rpd, lpd, flag):
    """Parameters of the plain cylinder at unit contrast (scale 1, no
    background); dispersity 35 points over 3 sigma when the width is > 0."""
    p = dict(radius=float(R), length=float(L), sld=1.0, sld_solvent=0.0,
             scale=1.0, background=0.0)
    if rpd > 0:
        p.update(radius_pd=float(rpd), radius_pd_n=PD_N, radius_pd_nsigma=3.0)
    if lpd > 0:
        p.update(length_pd=float(lpd), length_pd_n=PD_N, length_pd_nsigma=3.0)
    if not flag:
        p.update(theta=90.0, phi=0.0)
    return p


def model_columns(sets, idx, flag):
    """`model_pars` of the sets `idx` as parameter columns (a width of 0
    leaves the parameter without dispersity, as model_pars omits it)."""
    cols = dict(radius=np.asarray(sets["radius"], float)[idx],
                length=np.asarray(sets["length"], float)[idx], sld=1.0, sld_solvent=0.0,
                scale=1.0, background=0.0,
                radius_pd=np.maximum(np.asarray(sets["rpd"], float)[idx], 0.0),
                radius_pd_n=PD_N, radius_pd_nsigma=3.0,
                length_pd=np.maximum(np.asarray(sets["lpd"], float)[idx], 0.0),
                length_pd_n=PD_N, length_pd_nsigma=3.0)
    if not flag:
        cols.update(theta=90.0, phi=0.0)
    return cols


def plain_unit_iq(sets, qs, device=None, form="float32c", shape=None):
    """I(q) at unit contrast from the plain engines, one array per set, both
    through the batched engine: flag 1 as the 1D orientation average, flag 0
    as the 2D kernel at theta = 90, phi = 0 along qx (the line form, equal
    to Iqxy at q vectors (q, 0))."""
    from .batch import Population
    n = len(qs)
    out = [None]*n
    pops = []
    # both populations are packed and enqueued before either is read back,
    # so the host packing of the second overlaps the first one's kernels
    flags = np.asarray(sets["flag"]).astype(bool)
    for flag in (1, 0):
        idx = np.nonzero(flags == bool(flag))[0]
        if not idx.size:
            continue
        warps, ipw = (shape or {}).get(flag, (8, 8))
        pop = Population.from_columns("cylinder", [qs[k] for k in idx],
                                      model_columns(sets, idx, flag), form=form,
                                      device=device, line=not flag, warps=warps,
                                      items_per_warp=ipw)
        pop.run()
        pops.append((idx, pop))
    for idx, pop in pops:
        for k, iq in zip(idx, pop.iq()):
            out[k] = iq.copy()
    return out


def flatten(sets, qs):
    """Flat per-point arrays of (set parameters, q); "set" is the index of
    the parameter set each point belongs to."""
    counts = np.array([len(q) for q in qs])
    cols = {key: np.repeat(np.asarray(sets[key]), counts)
            for key in ("radius", "length", "rpd", "lpd", "contrast", "flag")}
    cols["q"] = np.concatenate(qs)
    cols["set"] = np.repeat(np.arange(len(qs)), counts)
    return cols


def envelope(err, set_id, window):
    """Running maximum of err over the `window` neighbours on each side
    within the same set (points of a set contiguous and sorted by q): the
    local error envelope, smooth where err itself crosses zero."""
    env = np.array(err, dtype=float, copy=True)
    sid = np.asarray(set_id)
    for s in range(1, window + 1):
        same = sid[s:] == sid[:-s]
        np.maximum(env[s:], np.where(same, err[:-s], 0.0), out=env[s:])
        np.maximum(env[:-s], np.where(same, err[s:], 0.0), out=env[:-s])
    return env


def gate_thresholds(r, err, tols, alpha):
    """For each tolerance, the largest threshold t on the gate's predicted
    error r such that among the points with r <= t at most a fraction
    `alpha` have err > tolerance (0 if no threshold qualifies); made
    non-decreasing in the tolerance."""
    order = np.argsort(r, kind="stable")
    rs, es = np.asarray(r)[order], np.asarray(err)[order]
    k = np.arange(1, len(rs) + 1)
    out = []
    for tol in tols:
        fine = np.flatnonzero(np.cumsum(es > tol) <= alpha*k)
        out.append(rs[fine[-1]] if len(fine) else 0.0)
    return np.maximum.accumulate(np.array(out, dtype=float))


class TrainingGraph:
    """One training step of an :class:`MLP` captured as a CUDA graph: the
    batch gather (rows named by ``idx``), the weight images, forward,
    loss, backward, weight gradients, the learning-rate schedule and Adam
    for every parameter; the schedule's counters live on the device, so a
    replay needs only the new row indices.  Launching the ~30 kernels of a
    step from Python costs more host time than their device time at batch
    8192; a replay costs one graph launch."""

    def __init__(self, net, x_all, x_lo_all, y_all, batch, lr, total, step0, warmup,
                 b1, b2, eps):
        torch = net.torch
        self.net = net
        dev = net.device
        if batch % TM:
            raise ValueError("batch must be a multiple of %d" % TM)
        self.batch = batch
        self.idx = torch.zeros(batch, dtype=torch.int64, device=dev)
        self.counters = torch.tensor([int(step0), int(net.step_count)], dtype=torch.int32,
                                     device=dev)
        self.sched = torch.zeros(4, dtype=torch.float32, device=dev)
        self.xb = torch.empty((batch, x_all.shape[1]), dtype=x_all.dtype, device=dev)
        self.xlb = torch.empty_like(self.xb)
        self.yb = torch.empty(batch, dtype=y_all.dtype, device=dev)
        net._scratch(batch)
        lib, st = net.lib, net.stream.cuda_stream
        net.stream.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=net.stream):
            torch.index_select(x_all, 0, self.idx, out=self.xb)
            torch.index_select(x_lo_all, 0, self.idx, out=self.xlb)
            torch.index_select(y_all, 0, self.idx, out=self.yb)
            net._check(lib.sasb200_lr_schedule(self.counters.data_ptr(), self.sched.data_ptr(),
                                               int(total), int(warmup), float(lr), b1, b2, st),
                       "lr_schedule")
            net._pack_kernels()
            self.loss, dW, db, gw, gbo = net._gradient_kernels(self.xb, self.xlb, self.yb, batch)
            grads = dW + db + [gw, gbo]
            nt = len(net.params)
            I32, VP = ct.c_int32*nt, ct.c_void_p*nt
            sizes = [p.numel() for p in net.params]
            splits = [net.splits if k < 4 else 1 for k in range(nt)]
            shape = [(HID, NIN if k == 0 else HID) if k < 4 else (0, 0) for k in range(nt)]
            net._check(lib.sasb200_adam_multi(
                nt, I32(*sizes), I32(*splits), VP(*[g.data_ptr() for g in grads]),
                VP(*[p.data_ptr() for p in net.params]), VP(*[m.data_ptr() for m in net.m]),
                VP(*[v.data_ptr() for v in net.v]),
                VP(*[net.Wb[k].data_ptr() if k < 4 else None for k in range(nt)]),
                VP(*[net.WTb[k].data_ptr() if k < 4 else None for k in range(nt)]),
                I32(*[r for r, _ in shape]), I32(*[c for _, c in shape]),
                self.sched.data_ptr(), b1, b2, eps, st), "adam_multi")

    def step(self, idx):
        """One training step on rows `idx` (int64 device tensor of `batch`
        entries); returns the loss (a device scalar, overwritten by the
        next step)."""
        net = self.net
        with net.torch.cuda.stream(net.stream):
            self.idx.copy_(idx)
            self.graph.replay()
        net.step_count += 1
        return self.loss


class Surrogate:
    """Trained network, its error gate, target scalings and the gate's
    calibrated thresholds."""

    TOL = 0.01
    #: tolerances (|log I error|) at which the gate is calibrated
    CAL_TOLS = np.unique(np.r_[np.logspace(-3, 0, 31), 0.01, 0.05])

    def __init__(self, device=None, seed=0):
        self.net = MLP(device=device, seed=seed)
        self.torch = self.net.torch
        self.seed = seed
        self.y_mean = 0.0
        self.y_std = 1.0
        self.gate = None
        self.g_mean = 0.0
        self.g_std = 1.0
        self.cal_tols = None
        self.cal_thresh = None
        self.alpha = None
        self.floor = 1e-5
        #: launch shape (warps, items per warp) of the batched fallback per
        #: orientation flag; None = the library default (8, 8)
        self.fallback_shape = None

    # ---- data --------------------------------------------------------------
    def dataset(self, n_sets, nq, seed, form="float32c", low_pd_frac=0.0):
        rng = np.random.default_rng(seed)
        sets = sample_sets(n_sets, rng, low_pd_frac=low_pd_frac)
        qs = [sample_q(nq, rng) for _ in range(n_sets)]
        iq = plain_unit_iq(sets, qs, self.net.device, form)
        cols = flatten(sets, qs)
        y = np.log(np.concatenate(iq))
        return cols, y

    def _x(self, cols):
        return self.net.features(cols["radius"], cols["length"], cols["rpd"], cols["lpd"],
                                 cols["contrast"], cols["q"], cols["flag"].astype(float))

    # ---- training ----------------------------------------------------------
    def _train(self, net, x_all, xlo_all, t_all, n, epochs, batch, lr, seed, scale, log, what,
               group=None):
        """Adam with cosine decay over shuffled batches of one network, all
        on its stream; returns the loss per epoch (in target units).

        Given a process group of several ranks (every rank holding the same
        training arrays and the same seed), each global batch is split into
        equal contiguous slices, one per rank, and the gradients averaged by
        one all-reduce per step: data-parallel replicas of the same run."""
        from .multigpu import allreduce_mean, batch_slice, broadcast_parameters
        torch = self.torch
        dist = torch.distributed
        nranks, rank, reduce = 1, 0, None
        if group is not None:
            nranks, rank = dist.get_world_size(group), dist.get_rank(group)
        if nranks > 1:
            broadcast_parameters(net, 0, group)

            def reduce(grads):
                allreduce_mean(grads, group)
        # the epochs' row orders come from a seeded generator on the device
        # (every replica of a data-parallel run draws the same ones)
        gen = torch.Generator(device=net.device)
        gen.manual_seed(int(seed))
        steps = max(1, n//batch)
        total = epochs*steps
        step = 0
        losses = []
        # on one GPU the first step runs eagerly (every kernel loaded), the
        # rest replay a CUDA graph of the step with the same schedule
        graph = None
        use_graph = nranks == 1 and (batch//nranks) % TM == 0
        for ep in range(epochs):
            perm = torch.randperm(n, device=net.device, generator=gen)
            for s in range(steps):
                lo, hi = batch_slice(s*batch, batch, rank, nranks)
                idx = perm[lo:hi]
                if graph is not None:
                    loss = graph.step(idx)
                    step += 1
                    continue
                with torch.cuda.stream(net.stream):
                    xb = x_all.index_select(0, idx)
                    xlb = xlo_all.index_select(0, idx)
                    tb = t_all.index_select(0, idx)
                # cosine decay with a short warm-up
                frac = step/total
                rate = lr*min(1.0, (step + 1)/WARMUP_STEPS)*0.5*(1 + math.cos(math.pi*frac))
                loss = net.train_step(xb, xlb, tb, hi - lo, rate, reduce=reduce)
                step += 1
                if use_graph and step < total:
                    graph = net.capture_training(x_all, xlo_all, t_all, hi - lo, lr, total, step,
                                                 warmup=WARMUP_STEPS)
            net.stream.synchronize()
            losses.append(float(loss.item())*scale**2)
            if log:
                log("%s epoch %d loss %.3e" % (what, ep, losses[-1]))
        graph = None
        if net.errors():
            raise RuntimeError("tensor-core kernel reported a timeout")
        return losses

    def fit(self, cols, y, epochs=8, batch=8192, lr=2e-3, seed=0, log=None, huber=0.05,
            group=None):
        """Train the network on log I at unit contrast (Huber loss with
        threshold `huber` in log I); data-parallel over the ranks of
        `group` (e.g. ``torch.distributed.group.WORLD``) when given."""
        torch = self.torch
        good = np.isfinite(y)
        cols = {k: v[good] for k, v in cols.items()}
        y = y[good]
        self.y_mean = float(y.mean())
        self.y_std = float(y.std())
        self.net.huber = huber/self.y_std
        x_all, xlo_all, n = self._x(cols)
        t_all = torch.as_tensor((y - self.y_mean)/self.y_std, dtype=torch.float32,
                                device=self.net.device)
        return self._train(self.net, x_all, xlo_all, t_all, n, epochs, batch, lr, seed,
                           self.y_std, log, "net", group)

    def fit_gate(self, cols, y, epochs=16, batch=8192, lr=2e-3, seed=0, log=None, huber=1.0,
                 window=16, group=None):
        """Train the error gate: a second network of the same shape (the same
        tensor-core kernels) that predicts log(envelope + floor) of the
        trained network's |log I error| from the same features, on sets the
        network has not seen; the envelope is the running maximum over
        `window` neighbouring q of the set on each side (the error itself
        crosses zero between them, which no smooth predictor can follow).
        Returns the per-point errors."""
        torch = self.torch
        good = np.isfinite(y)
        cols = {k: v[good] for k, v in cols.items()}
        y = y[good]
        logi, _ = self._outputs(cols, gate=False)
        err = np.abs(logi - 2.0*np.log(np.abs(cols["contrast"])) - y)
        target = np.log(envelope(err, cols["set"], window) + self.floor)
        self.g_mean = float(target.mean())
        self.g_std = float(target.std())
        self.gate = MLP(device=self.net.device, seed=self.seed + 7919, stream=self.net.stream)
        self.gate.huber = huber/self.g_std
        x_all, xlo_all, n = self._x(cols)
        t_all = torch.as_tensor((target - self.g_mean)/self.g_std, dtype=torch.float32,
                                device=self.net.device)
        self._train(self.gate, x_all, xlo_all, t_all, n, epochs, batch, lr, seed + 1,
                    self.g_std, log, "gate", group)
        return err

    # ---- inference ----------------------------------------------------------
    def _outputs(self, cols, gate=True):
        """(predicted log I with the contrast, gate output or None) for flat
        arrays of inputs: one feature pass, both networks through the
        inference kernel."""
        torch = self.torch
        x, x_lo, n = self._x(cols)
        with torch.cuda.stream(self.net.stream):
            out = self.net.serve(x, x_lo, n)[:n].double()*self.y_std + self.y_mean
            g = None
            if gate and self.gate is not None:
                g = self.gate.serve(x, x_lo, n)[:n].double()*self.g_std + self.g_mean
            out = out.cpu()
            g = g.cpu() if g is not None else None
        self.net.stream.synchronize()
        logc = 2.0*np.log(np.abs(cols["contrast"]))
        return out.numpy() + logc, (g.numpy() if g is not None else None)

    def predict_log(self, cols):
        """Predicted log I (with the contrast) for flat arrays of inputs."""
        return self._outputs(cols, gate=False)[0]

    @staticmethod
    def inside(cols):
        """Points inside the training domain (with a nonzero contrast)."""
        ok = np.ones(len(cols["q"]), bool)
        for key in ("radius", "length", "rpd", "lpd", "contrast", "q"):
            lo, hi = DOMAIN[key]
            ok &= (cols[key] >= lo) & (cols[key] <= hi)
        return ok & (np.abs(cols["contrast"]) > 0)

    def _predicted(self, cols, g):
        """Smallest calibrated tolerance at which each point is accepted."""
        n = len(cols["q"])
        if g is None or self.cal_thresh is None:
            return np.full(n, np.inf)
        r = np.exp(g)
        # thresholds grow with the tolerance: first k with r <= thresh[k]
        k = np.searchsorted(self.cal_thresh, r, side="left")
        pe = np.where(k < len(self.cal_tols),
                      self.cal_tols[np.minimum(k, len(self.cal_tols) - 1)], np.inf)
        return np.where(self.inside(cols), pe, np.inf)

    def predicted_error(self, cols):
        """Predicted |log I error| per point: the smallest calibrated
        tolerance whose gate threshold admits the point; infinite outside the
        training domain or before calibration."""
        return self._predicted(cols, self._outputs(cols)[1])

    def calibrate(self, cols, y_true, alpha=5e-4):
        """Calibrate the gate on held-out sets judged by the plain FP64
        kernel: for each tolerance in CAL_TOLS, the largest threshold on
        exp(gate) for which at most a fraction `alpha` of the accepted
        points are in fact off by more than that tolerance.  Returns the
        per-point errors."""
        logi, g = self._outputs(cols)
        err = np.abs(logi - 2.0*np.log(np.abs(cols["contrast"])) - y_true)
        ok = self.inside(cols) & np.isfinite(err)
        self.cal_thresh = gate_thresholds(np.exp(g[ok]), err[ok], self.CAL_TOLS, alpha)
        self.cal_tols = self.CAL_TOLS.copy()
        self.alpha = alpha
        return err

    def _accept_log_threshold(self, tol):
        """log of the gate threshold at tolerance `tol` (the largest
        calibrated tolerance not above it); -inf when nothing is trusted."""
        if self.gate is None or self.cal_thresh is None:
            return -np.inf
        k = np.searchsorted(self.cal_tols, tol, side="right") - 1
        if k < 0 or self.cal_thresh[k] <= 0:
            return -np.inf
        return float(np.log(self.cal_thresh[k]))

    def _device_eval(self, cols, tol):
        """(I, accepted mask) of the network at every point, computed on the
        device: only q, a run index and one row per run of points sharing a
        parameter set cross to the GPU (points of a set are contiguous, as
        flatten() lays them out); the domain check, the gate threshold and
        exp(log I) run there too."""
        torch = self.torch
        dev = self.net.device
        sid = np.asarray(cols["set"])
        n = len(sid)
        new = np.r_[True, sid[1:] != sid[:-1]] if n else np.zeros(0, bool)
        starts = np.flatnonzero(new)
        run = (np.cumsum(new) - 1).astype(np.int32)
        keys = ("radius", "length", "rpd", "lpd", "contrast", "flag")
        table = np.stack([np.asarray(cols[k], float)[starts] for k in keys], axis=1)
        ok = np.abs(table[:, 4]) > 0
        for j, key in enumerate(keys[:5]):
            lo, hi = DOMAIN[key]
            ok &= (table[:, j] >= lo) & (table[:, j] <= hi)
        table = np.concatenate([table, ok[:, None].astype(float)], axis=1)
        thr = self._accept_log_threshold(tol)
        qlo, qhi = DOMAIN["q"]
        with torch.cuda.stream(self.net.stream):
            T = torch.as_tensor(table, device=dev).index_select(
                0, torch.as_tensor(run, device=dev))
            q = torch.as_tensor(np.ascontiguousarray(cols["q"], 'd'), device=dev)
            x, x_lo, _ = self.net.features(T[:, 0], T[:, 1], T[:, 2], T[:, 3], T[:, 4], q,
                                           T[:, 5])
            logi = (self.net.serve(x, x_lo, n)[:n].double()*self.y_std + self.y_mean
                    + 2.0*torch.log(T[:, 4].abs()))
            accept = (T[:, 6] > 0.5) & (q >= qlo) & (q <= qhi)
            if np.isfinite(thr):
                g = self.gate.serve(x, x_lo, n)[:n].double()*self.g_std + self.g_mean
                accept &= g <= thr
            else:
                accept &= False
            I = torch.exp(logi).cpu().numpy()
            acc = accept.cpu().numpy()
        return I, acc

    def iq(self, cols, tol=None, device=None, form="float32c"):
        """I(q) for flat inputs: the network where its predicted error is
        within `tol` (log I), the plain kernel elsewhere (its FP32c form by
        default, within 1e-5 of FP64, far inside the tolerance).  Returns
        (I, mask of points that fell back)."""
        tol = self.TOL if tol is None else tol
        I, accepted = self._device_eval(cols, tol)
        back = ~accepted
        if back.any():
            I[back] = self.plain(cols, back, device, form)
        return I, back

    def plain(self, cols, mask, device=None, form="double"):
        """Plain-kernel I(q) (with contrast) at the masked points, one plain
        evaluation per parameter set over just its masked q."""
        idx = np.nonzero(mask)[0]
        sid = cols["set"][idx]
        order = np.argsort(sid, kind="stable")
        idx, sid = idx[order], sid[order]
        starts = np.flatnonzero(np.r_[True, sid[1:] != sid[:-1]])
        ends = np.r_[starts[1:], len(sid)]
        first = idx[starts]
        sets = {k: cols[k][first] for k in ("radius", "length", "rpd", "lpd", "contrast",
                                            "flag")}
        sets["flag"] = sets["flag"].astype(int)
        qs = [cols["q"][idx[a:b]] for a, b in zip(starts, ends)]
        iq = plain_unit_iq(sets, qs, device or self.net.device, form,
                           shape=self.fallback_shape if form == "float32c" else None)
        vals = np.empty(len(idx))
        for (a, b), v, c in zip(zip(starts, ends), iq, sets["contrast"]):
            vals[a:b] = v*c*c
        out = np.empty(len(mask))
        out[idx] = vals
        return out[mask]

    def save(self, path):
        st = self.net.state()
        extra = {}
        if self.gate is not None:
            gs = self.gate.state()
            extra = dict(**{"gW%d" % l: gs["W"][l] for l in range(4)},
                         **{"gb%d" % l: gs["b"][l] for l in range(4)},
                         g_w_out=gs["w_out"], g_b_out=gs["b_out"])
        if self.cal_thresh is not None:
            extra.update(cal_tols=self.cal_tols, cal_thresh=self.cal_thresh)
        np.savez(path, y_mean=self.y_mean, y_std=self.y_std, g_mean=self.g_mean,
                 g_std=self.g_std, floor=self.floor,
                 **{"W%d" % l: st["W"][l] for l in range(4)},
                 **{"b%d" % l: st["b"][l] for l in range(4)},
                 w_out=st["w_out"], b_out=st["b_out"], **extra)

    def load(self, path):
        d = np.load(path)
        self.y_mean = float(d["y_mean"])
        self.y_std = float(d["y_std"])
        self.net.load_state({"W": [d["W%d" % l] for l in range(4)],
                             "b": [d["b%d" % l] for l in range(4)],
                             "w_out": d["w_out"], "b_out": d["b_out"]})
        if "gW0" in d:
            self.g_mean, self.g_std = float(d["g_mean"]), float(d["g_std"])
            self.floor = float(d["floor"])
            self.gate = MLP(device=self.net.device, seed=self.seed + 7919,
                            stream=self.net.stream)
            self.gate.load_state({"W": [d["gW%d" % l] for l in range(4)],
                                  "b": [d["gb%d" % l] for l in range(4)],
                                  "w_out": d["g_w_out"], "b_out": d["g_b_out"]})
        if "cal_thresh" in d:
            self.cal_tols, self.cal_thresh = d["cal_tols"], d["cal_thresh"]


def train_and_evaluate(n_train_sets=50000, nq=1000, epochs=10, n_holdout_sets=1000,
                       batch=8192, lr=2e-3, tol=0.01, seed=0, device=None, log=None,
                       data_form="float32c", low_pd_frac=0.4, n_gate_sets=None,
                       gate_epochs=16, alpha=5e-4):
    """
    Generate training data with the plain kernels and train the network;
    train the error gate on fresh sets; on held-out sets judged by the plain
    FP64 kernels, calibrate the gate thresholds (two thirds) and measure (one
    third): accuracy, and the throughput of the surrogate with automatic
    fallback against the plain FP64 (and FP32c) path on the same points.
    """
    import time
    import torch
    say = log or (lambda *a: None)
    S = Surrogate(device=device, seed=seed)
    t0 = time.perf_counter()
    cols, y = S.dataset(n_train_sets, nq, seed + 1, form=data_form, low_pd_frac=low_pd_frac)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    say("data: %d samples in %.1f s" % (len(y), t_data))
    t0 = time.perf_counter()
    losses = S.fit(cols, y, epochs=epochs, batch=batch, lr=lr, seed=seed, log=say)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del cols, y
    # error gate on sets the network has not seen (FP32c labels: within 1e-5,
    # far inside the tolerances)
    if n_gate_sets is None:
        n_gate_sets = max(n_train_sets//5, 300)
    t0 = time.perf_counter()
    gcols, gy = S.dataset(n_gate_sets, nq, seed + 3, form=data_form, low_pd_frac=low_pd_frac)
    S.fit_gate(gcols, gy, epochs=gate_epochs, batch=batch, lr=lr, seed=seed, log=say)
    torch.cuda.synchronize()
    t_gate = time.perf_counter() - t0
    del gcols, gy
    rng = np.random.default_rng(seed + 2)
    sets = sample_sets(n_holdout_sets, rng)
    qs = [sample_q(nq, rng) for _ in range(n_holdout_sets)]
    half = (2*n_holdout_sets)//3
    cal = ({k: v[:half] for k, v in sets.items()}, qs[:half])
    ev = ({k: v[half:] for k, v in sets.items()}, qs[half:])
    cal_cols = flatten(*cal)
    cal_y = np.log(np.concatenate(plain_unit_iq(cal[0], cal[1], S.net.device, "double")))
    S.calibrate(cal_cols, cal_y, alpha=alpha)
    ev_cols = flatten(*ev)
    # plain FP64 path on the measured part (also the ground truth), and the
    # plain FP32c path for reference; one untimed call of each first
    plain_unit_iq({k: v[:8] for k, v in ev[0].items()}, ev[1][:8], S.net.device, "double")
    plain_unit_iq({k: v[:8] for k, v in ev[0].items()}, ev[1][:8], S.net.device, "float32c")
    # every arm below is timed on the host clock as the mean of REPS calls,
    # so that one stall of the host does not decide a ratio
    REPS = 3

    def timed(fn):
        out, total = None, 0.0
        for _ in range(REPS):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            total += time.perf_counter() - t0
        return out, total/REPS
    ev_iq, t_plain = timed(lambda: plain_unit_iq(ev[0], ev[1], S.net.device, "double"))
    _, t_plain32 = timed(lambda: plain_unit_iq(ev[0], ev[1], S.net.device, "float32c"))
    truth = np.log(np.concatenate(ev_iq)) + 2*np.log(np.abs(ev_cols["contrast"]))
    S.predict_log(ev_cols)            # warm
    _, t_net = timed(lambda: S.predict_log(ev_cols))
    logi, g = S._outputs(ev_cols)
    raw = np.abs(logi - truth)
    n = len(truth)
    report = dict(
        train_samples=int(n_train_sets*nq), epochs=epochs, data_s=t_data, train_s=t_train,
        gate_samples=int(n_gate_sets*nq), gate_epochs=gate_epochs, gate_s=t_gate,
        gate_alpha=alpha, final_loss=losses[-1], holdout_samples=int(n),
        net_median_err=float(np.median(raw)), net_p90_err=float(np.quantile(raw, 0.9)),
        net_p99_err=float(np.quantile(raw, 0.99)),
        plain_samples_per_s=n/t_plain, plain_f32c_samples_per_s=n/t_plain32,
        net_only_samples_per_s=n/t_net,
        net_only_speedup=t_plain/t_net, operating_points={})
    # surrogate with automatic fallback, timed end to end, at each tolerance
    # (one untimed call of each first: module loading, allocator warm-up)
    for t in sorted({tol, 0.05}):
        S.iq(ev_cols, tol=t)
    for t in sorted({tol, 0.05}):
        (I, back), t_sur = timed(lambda: S.iq(ev_cols, tol=t))
        err = np.abs(np.log(I) - truth)
        report["operating_points"]["%g" % t] = dict(
            net_frac_within=float(np.mean(raw <= t)), fallback_frac=float(back.mean()),
            frac_within=float(np.mean(err <= t)),
            accepted_frac_within=float(np.mean(err[~back] <= t)) if (~back).any() else 1.0,
            max_err=float(err.max()), samples_per_s=n/t_sur, speedup=t_plain/t_sur,
            speedup_vs_plain_f32c=t_plain32/t_sur)
    return S, report
