"""
CPU oracle for the surrogate MLP (test infrastructure only).

numpy restatement of the forward and backward passes of the tensor-core MLP
in ``sasmodels_b200/csrc/mlp.cu``: 16 -> 256 -> 256 -> 256 -> 256 -> 1,
SiLU, z = h W^T + b, out = h3 . w_out + b_out, MSE loss.  With
``emulate_bf16=True`` every value the GPU stores as BF16 (weights, saved
z/h, dZ; inputs and hidden activations as a compensated hi + lo BF16 pair) is
rounded the same way, so the device gradients can be compared tightly; with ``False`` it is
the plain FP64 mathematics the kernels approximate.  SiLU and its derivative here are exact;
the kernels take the sigmoid in both as (1 + tanh(z/2))/2 with the hardware tanh
approximation (relative error about 2^-11), which the tests' tolerances cover.
"""

import numpy as np


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def silu(z):
    return z/(1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0/(1.0 + np.exp(-z))
    return s*(1.0 + z*(1.0 - s))


def split_bf16(a):
    """Compensated BF16 pair hi + lo of a, summed (what the kernels feed the
    tensor cores as two BF16 operands)."""
    hi = bf16(a)
    return hi + bf16(np.asarray(a, np.float64) - hi)


def forward(x, W, b, w_out, b_out, emulate_bf16=True, split_act=True):
    """Returns out and the saved (z, h) per hidden layer.  With
    ``split_act`` the layer inputs carry the compensated hi + lo pair."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    feed = split_bf16 if (emulate_bf16 and split_act) else r
    a = feed(x)
    zs, hs = [], []
    for l in range(4):
        z = a @ r(W[l]).T + b[l]
        h = silu(z)
        zs.append(r(z))
        hs.append(r(h))
        a = feed(h)
        last_h = h
    out = last_h @ w_out + b_out
    return out, zs, hs


def backward(x, W, w_out, dout, zs, hs, emulate_bf16=True):
    """Gradients of sum(dout * out) w.r.t. W[l], b[l], w_out, b_out, using
    the saved z and h of :func:`forward`."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    dz = [None]*4
    dz[3] = r(dout[:, None]*w_out[None, :]*dsilu(zs[3]))
    for l in range(3, 0, -1):
        dh = dz[l] @ r(W[l])
        dz[l - 1] = r(dh*dsilu(zs[l - 1]))
    inputs = [r(x)] + [hs[l] for l in range(3)]
    dW = [dz[l].T @ inputs[l] for l in range(4)]
    db = [dz[l].sum(axis=0) for l in range(4)]
    dw_out = hs[3].T @ dout
    db_out = dout.sum()
    return dW, db, dw_out, db_out
