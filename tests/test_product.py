"""
P@S products (sasmodels_b200.product) against the reference's own product
machinery recorded in tests/golden/product.json (make_product_golden.py):
the combined parameter table and marshaling on the CPU, bitwise; the device
chain (P sums -> S values patched on the device -> S -> combination) on the
GPU against the reference ProductKernel over its DLLs, within 1e-12.
"""

import json
import os

import numpy as np
import pytest

from helpers import GOLDEN

with open(os.path.join(GOLDEN, "product.json")) as _fid:
    CASES = json.load(_fid)

#: Below q = LOW_Q the structure factors of these products are evaluated by
#: the reference (and here) through closed forms whose terms cancel to about
#: 1e-6 of their size just above the small-qR series cut-off (hardsphere.c
#: uses its series only for 2 q R_eff < 0.05; squarewell.c and the
#: Hayter-Penfold MSA solve behave alike), so a one-ulp difference between
#: CUDA's and glibc's sin/cos/exp comes out at up to ~3e-9 relative.  The
#: inputs handed to S (R_eff, volume fraction x volume ratio) equal the
#: DLL's bit for bit (test_gpu_parity.py::test_norms_in_dll_order).
PRODUCT_RTOL = 5e-9
LOW_Q = 0.02


@pytest.mark.parametrize("k", range(len(CASES)))
def test_product_table_and_marshal(k):
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    c = CASES[k]
    info = load_model_info(c["name"])
    assert [p.name for p in info.parameters.call_parameters] == c["call_parameters"]
    qv = [np.array(v) for v in c["q"]]
    details, values, _ = make_call_args(info, c["pars"], qv)
    np.testing.assert_array_equal(details.buffer, c["details"])
    np.testing.assert_array_equal(values, c["values"])


def test_product_rejects_bad_structure_factor():
    from sasmodels_b200.core import load_model_info
    with pytest.raises(TypeError):
        load_model_info("sphere@cylinder")


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(len(CASES)))
def test_product_gpu(cuda, k):
    from sasmodels_b200 import load_model
    from sasmodels_b200.direct_model import call_kernel
    c = CASES[k]
    model = load_model(c["name"])
    qv = [np.array(v) for v in c["q"]]
    kernel = model.make_kernel(qv)
    I = call_kernel(kernel, dict(c["pars"]))
    ref = np.array(c["I"])
    rel = np.abs(I - ref)/np.abs(ref)
    qmag = np.sqrt(sum(np.array(v)**2 for v in c["q"]))
    # the structure factors' closed forms cancel at small q R_eff (see
    # PRODUCT_RTOL); elsewhere the product meets the FP64 bar
    assert rel.max() <= PRODUCT_RTOL, (c["name"], rel.max())
    well = qmag > LOW_Q
    assert rel[well].max() <= 1e-12, (c["name"], rel[well].max(), qmag[well][np.argmax(rel[well])])
    # a second call reuses the kernels and buffers
    np.testing.assert_allclose(call_kernel(kernel, dict(c["pars"])), I, rtol=0, atol=0)
