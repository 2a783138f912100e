"""
The allocation-free entry point, sasb200_cylinder_Iqxy_noalloc.

It exists for callers that may not allocate GPU memory themselves (plugins
inside another program's CUDA context, code running under that program's
allocator lock, real-time loops), so it takes its scratch from a fixed 8 MiB
device array instead of a caller workspace.  These tests call it through the
C-ABI and check it against the regular workspace entry point on two calls in
a row (the scratch keeps the previous call's contents, which must not leak
into the next result), against the reference DLL on a block of the grid
where the asymptotic J1 branch runs, with an effective radius requested
(per-point norm terms, whose stride changes with the chunk), on a restarted
mesh (pd_start > 0 adds to the result), plus the size rejection.  The file
name makes pytest collect it last.
"""

import ctypes as ct

import numpy as np
import pytest

from helpers import RTOL_FP64, compare_raw, load_info, marshal, reference_raw
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


def _case(n, reff_mode=0, **mesh):
    import torch
    name, qv, pars = workloads.cylinder_2d(n=n, **mesh)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    with torch.cuda.stream(kernel.stream):
        ref = kernel.launch("Iqxy", dev_d, dev_v, 0, details.num_eval, 0.0,
                            reff_mode).clone()
    kernel.stream.synchronize()
    return kernel, details, dev_d, dev_v, ref.cpu().numpy()


def _call(fn, err, kernel, dev_d, dev_v, pd_start, pd_stop, out, reff_mode=0):
    status = fn(kernel.q_input.nq, pd_start, pd_stop, dev_d.data_ptr(), dev_v.data_ptr(),
                kernel.q_input.q_dev.data_ptr(), out.data_ptr(), 0.0, reff_mode, 0,
                kernel.stream.cuda_stream)
    assert status == 0, err().decode()
    kernel.stream.synchronize()
    return out.cpu().numpy()


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


def test_noalloc_against_reference_dll(cuda):
    """The corner 8x8 block of the 256x256 cylinder grid at the full
    490000-point mesh (more than half of its evaluations take the asymptotic
    J1 branch), through the allocation-free entry point, against the
    reference DLL on the same inputs, on two calls in a row."""
    import torch
    fn, err = _noalloc_fn()
    name, qv, pars = workloads.cylinder_2d_subgrid(8, where="corner")
    assert workloads.cylinder_j1_large_fraction(qv[0], qv[1], pars) > 0.5
    model = load_model(name)
    kernel = model.make_kernel(qv, reorder=False)
    details, values, _ = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    nq = kernel.q_input.nq
    ref = reference_raw(name, load_info(name), qv, pars, threads=8)
    for _ in range(2):
        out = torch.full((nq + 4,), float("nan"), dtype=torch.float64, device=kernel.device)
        got = _call(fn, err, kernel, dev_d, dev_v, 0, details.num_eval, out)
        worst, f2rel = compare_raw(got, ref, 1, nq, RTOL_FP64)
        assert worst <= 1.0, (worst, f2rel)


def test_noalloc_effective_radius_chunked(cuda):
    """radius_effective_mode 1 on the chunked 490000-point mesh: the four norm
    sums are accumulated point by point in mesh order from per-point terms
    whose stride follows the chunk; they must equal the workspace entry
    point's bit for bit, and the F^2 slots must agree within the FP64 bar."""
    import torch
    fn, err = _noalloc_fn()
    kernel, details, dev_d, dev_v, ref = _case(8, reff_mode=1)
    nq = kernel.q_input.nq
    for _ in range(2):
        out = torch.full((nq + 4,), float("nan"), dtype=torch.float64, device=kernel.device)
        got = _call(fn, err, kernel, dev_d, dev_v, 0, details.num_eval, out, reff_mode=1)
        np.testing.assert_array_equal(got[nq:nq + 4], ref[nq:nq + 4])
        worst, f2rel = compare_raw(got, ref[:nq + 4], 1, nq, RTOL_FP64)
        assert worst <= 1.0, (worst, f2rel)


@pytest.mark.parametrize("reff_mode", [0, 1])
def test_noalloc_restarted_mesh(cuda, reff_mode):
    """pd_start > 0 continues a partly computed mesh: a call over
    [0, k) followed by one over [k, n) into the same result gives the
    single-call sums (the reference's restart contract), with the second
    call's first chunk adding to what the first call left."""
    import torch
    fn, err = _noalloc_fn()
    kernel, details, dev_d, dev_v, ref = _case(8, reff_mode=reff_mode)
    nq = kernel.q_input.nq
    n = details.num_eval
    k = 3*n//7 + 5                 # not on a segment or chunk boundary
    out = torch.full((nq + 4,), float("nan"), dtype=torch.float64, device=kernel.device)
    _call(fn, err, kernel, dev_d, dev_v, 0, k, out, reff_mode)
    got = _call(fn, err, kernel, dev_d, dev_v, k, n, out, reff_mode)
    worst, f2rel = compare_raw(got, ref[:nq + 4], 1, nq, RTOL_FP64)
    assert worst <= 1.0, (worst, f2rel)
    if reff_mode:
        np.testing.assert_array_equal(got[nq:nq + 4], ref[nq:nq + 4])
