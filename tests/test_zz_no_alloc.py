"""
The allocation-free entry point, sasb200_cylinder_Iqxy_noalloc.

It exists for callers that may not allocate GPU memory themselves (plugins
inside another program's CUDA context, code running under that program's
allocator lock, real-time loops), so it takes its scratch from a fixed 8 MiB
device array instead of a caller workspace.  These tests call it through the
C-ABI and check it against the regular workspace entry point on two calls in
a row (the scratch keeps the previous call's contents, which must not leak
into the next result), plus the size rejection.  The file name makes pytest
collect it last.
"""

import ctypes as ct

import numpy as np
import pytest

from helpers import RTOL_FP64, compare_raw, marshal
from sasmodels_b200 import _abi, load_model, workloads

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 8 << 20


def _noalloc_fn():
    lib = ct.CDLL(_abi.library_path("cylinder"))
    fn = lib.sasb200_cylinder_Iqxy_noalloc
    fn.argtypes = [ct.c_int32, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_void_p,
                   ct.c_void_p, ct.c_void_p, ct.c_double, ct.c_int32, ct.c_int32,
                   ct.c_void_p]
    fn.restype = ct.c_int32
    err = lib.sasb200_cylinder_last_error
    err.restype = ct.c_char_p
    return fn, err


def _case(n, **mesh):
    import torch
    name, qv, pars = workloads.cylinder_2d(n=n, **mesh)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    with torch.cuda.stream(kernel.stream):
        ref = kernel.launch("Iqxy", dev_d, dev_v, 0, details.num_eval, 0.0, 0).clone()
    kernel.stream.synchronize()
    return kernel, details, dev_d, dev_v, ref.cpu().numpy()


@pytest.mark.parametrize("n, mesh", [
    (24, dict(radius_n=9, length_n=7, theta_n=5, phi_n=5)),
    # 490000-point mesh: larger than one pass of the scratch, so it is chunked
    (8, {}),
])
def test_noalloc_matches_workspace_entry(cuda, n, mesh):
    import torch
    fn, err = _noalloc_fn()
    kernel, details, dev_d, dev_v, ref = _case(n, **mesh)
    nq = kernel.q_input.nq
    outs = []
    for _ in range(2):
        out = torch.full((nq + 4,), float("nan"), dtype=torch.float64,
                         device=kernel.device)
        status = fn(nq, 0, details.num_eval, dev_d.data_ptr(), dev_v.data_ptr(),
                    kernel.q_input.q_dev.data_ptr(), out.data_ptr(), 0.0, 0, 0,
                    kernel.stream.cuda_stream)
        assert status == 0, err().decode()
        kernel.stream.synchronize()
        outs.append(out.cpu().numpy())
    for out in outs:
        worst, f2rel = compare_raw(out, ref[:nq + 4], 1, nq, RTOL_FP64)
        assert worst <= 1.0, (worst, f2rel)
    # same tile, same chunking: the second call reproduces the first exactly
    np.testing.assert_array_equal(outs[0], outs[1])


def test_noalloc_rejects_oversized_problem(cuda):
    """A q count whose per-segment scratch exceeds the 8 MiB array is refused
    with a message, before any kernel runs."""
    fn, err = _noalloc_fn()
    nq = 2*SCRATCH_BYTES//8          # the partial sums alone exceed the array
    status = fn(nq, 0, 128, 1, 1, 1, 1, 0.0, 0, 0, None)
    assert status == -2
    assert "static scratch" in err().decode()
