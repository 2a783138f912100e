"""
Resolution smearing (sasmodels_b200.resolution) against the reference's own
Pinhole1D / Pinhole2D outputs recorded in tests/golden/resolution.json.

CPU: the oracle restatement reproduces the recorded results; the product's
host side (q_calc, bands, 2D oversampling points and weights) equals the
reference's; the 2D averaging order of the GPU kernel reproduces numpy's
bit for bit.  GPU: the smearing kernels against the recorded results (1D
within 1e-12, 2D bitwise), from host arrays and from device tensors, and a
fused model-kernel + smearing step against the reference DLL + dense matrix.
"""

import json
import os

import numpy as np
import pytest

from helpers import GOLDEN

with open(os.path.join(GOLDEN, "resolution.json")) as _fid:
    GOLD = json.load(_fid)


class _Data2D:
    def __init__(self, c):
        self.qx_data, self.qy_data = np.array(c["qx"]), np.array(c["qy"])
        self.q_data = np.sqrt(self.qx_data**2 + self.qy_data**2)
        self.dqx_data, self.dqy_data = np.array(c["dqx"]), np.array(c["dqy"])


@pytest.mark.parametrize("k", range(len(GOLD["pinhole1d"])))
def test_pinhole1d_host_and_oracle(k):
    from oracle import resolution_ref
    from sasmodels_b200.resolution import Pinhole1D
    c = GOLD["pinhole1d"][k]
    q, dq = np.array(c["q"]), np.array(c["dq"])
    r = Pinhole1D(q, dq)
    np.testing.assert_array_equal(r.q_calc, c["q_calc"])
    W = resolution_ref.pinhole_matrix(r._signed_q_calc, q, np.maximum(dq, 1e-8))
    got = resolution_ref.smear_1d(W, np.array(c["theory"]))
    np.testing.assert_allclose(got, c["result"], rtol=1e-14, atol=0)
    # the bands hold exactly the nonzero weights of the dense matrix
    for i in range(len(q)):
        nz = np.flatnonzero(W[:, i])
        assert nz[0] >= r.band_lo[i] and nz[-1] < r.band_hi[i]
    np.testing.assert_array_equal(r.weight_matrix, W)


@pytest.mark.parametrize("k", range(len(GOLD["pinhole2d"])))
def test_pinhole2d_host_and_order(k):
    from oracle import resolution_ref
    from sasmodels_b200.resolution import Pinhole2D
    c = GOLD["pinhole2d"][k]
    r = Pinhole2D(_Data2D(c), accuracy=c["accuracy"], coords=c["coords"])
    np.testing.assert_array_equal(r.q_calc[0], c["qx_calc"])
    np.testing.assert_array_equal(r.q_calc[1], c["qy_calc"])
    np.testing.assert_array_equal(r.q_calc_weights, c["weights"])
    th, w, nq = np.array(c["theory"]), np.array(c["weights"]), len(c["qx"])
    np.testing.assert_array_equal(resolution_ref.average_2d(th, w, nq), c["result"])
    # the kernel's order: products rounded, summed bin by bin, one division
    t = th.reshape(len(w), nq)
    num = t[0]*w[0]
    for b in range(1, len(w)):
        num = num + t[b]*w[b]
    wgt = np.broadcast_to(w, (1, len(w))).swapaxes(-1, 0).sum(axis=0)[0]
    np.testing.assert_array_equal(num/wgt, c["result"])


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(len(GOLD["pinhole1d"])))
def test_pinhole1d_gpu(cuda, k):
    import torch
    from sasmodels_b200.resolution import Pinhole1D
    c = GOLD["pinhole1d"][k]
    r = Pinhole1D(np.array(c["q"]), np.array(c["dq"]))
    th = np.array(c["theory"])
    np.testing.assert_allclose(r.apply(th), c["result"], rtol=1e-12, atol=0)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        dev = torch.as_tensor(th, device="cuda")
        out = r.apply(dev, stream=st)
    st.synchronize()
    assert out.is_cuda
    np.testing.assert_allclose(out.cpu().numpy(), c["result"], rtol=1e-12, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(len(GOLD["pinhole2d"])))
def test_pinhole2d_gpu_bitwise(cuda, k):
    from sasmodels_b200.resolution import Pinhole2D
    c = GOLD["pinhole2d"][k]
    r = Pinhole2D(_Data2D(c), accuracy=c["accuracy"], coords=c["coords"])
    np.testing.assert_array_equal(r.apply(np.array(c["theory"])), c["result"])


@pytest.mark.gpu
def test_fused_model_and_smearing(cuda):
    """Sphere I(q_calc) left on the device by the kernel, smeared there,
    against the reference DLL's I(q_calc) times the dense matrix."""
    import torch
    from helpers import load_info, marshal, normalise, reference_raw
    from oracle import resolution_ref
    from sasmodels_b200 import load_model
    from sasmodels_b200.resolution import Pinhole1D
    q = np.logspace(-3, np.log10(0.5), 200)
    res = Pinhole1D(q, 0.08*q)
    pars = dict(radius=50, radius_pd=0.1, radius_pd_n=35, sld=4, sld_solvent=1,
                background=0.001)
    model = load_model("sphere")
    kernel = model.make_kernel([res.q_calc])
    details, values, magnetic = marshal(model.info, pars, [res.q_calc])
    dd, dv = kernel.upload(details, values)
    I_calc = kernel.Iq_device(dd, dv, details.num_eval, values[0], values[1])
    smeared = res.apply(I_calc, stream=kernel.stream)
    kernel.stream.synchronize()
    info = load_info("sphere")
    raw = reference_raw("sphere", info, [res.q_calc], pars)
    I_ref = normalise(raw, 2, len(res.q_calc), values)["I"]
    W = resolution_ref.pinhole_matrix(res._signed_q_calc, q, 0.08*q)
    np.testing.assert_allclose(smeared.cpu().numpy(), resolution_ref.smear_1d(W, I_ref),
                               rtol=1e-12, atol=0)


@pytest.mark.parametrize("k", range(len(GOLD["slit1d"])))
def test_slit1d_host_and_oracle(k):
    from oracle import resolution_ref
    from sasmodels_b200.resolution import Slit1D
    c = GOLD["slit1d"][k]
    q = np.array(c["q"])
    r = Slit1D(q, q_length=c["q_length"], q_width=c["q_width"])
    np.testing.assert_array_equal(r.q_calc, c["q_calc"])
    W = resolution_ref.slit_matrix(r._signed_q_calc, q, r._length, r._width)
    got = resolution_ref.smear_1d(W, np.array(c["theory"]))
    np.testing.assert_allclose(got, c["result"], rtol=1e-14, atol=0)


def test_slit1d_refuses_width_without_length():
    from sasmodels_b200.resolution import Slit1D
    with pytest.raises(NotImplementedError):
        Slit1D(np.linspace(0.01, 0.1, 10), q_length=0.0, q_width=0.01)


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(len(GOLD["slit1d"])))
def test_slit1d_gpu(cuda, k):
    from sasmodels_b200.resolution import Slit1D
    c = GOLD["slit1d"][k]
    r = Slit1D(np.array(c["q"]), q_length=c["q_length"], q_width=c["q_width"])
    np.testing.assert_allclose(r.apply(np.array(c["theory"])), c["result"], rtol=1e-12, atol=0)
