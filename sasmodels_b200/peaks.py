"""
Measured FP64 / FP32 / transcendental-unit throughput of the current GPU.

The sasmodels kernels are arithmetic bound on the FP64 pipe (FP64 form) or on
FP32 FMA and the MUFU unit (FP32 forms), so their roofline denominators are
measured here with the probes of ``csrc/peaks.cu``, timed with CUDA events
on the launching stream after warm-up.
"""

import ctypes as ct
import os

from ._abi import LIB_DIR

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(LIB_DIR, "libsasb200_peaks.so")
        if not os.path.exists(path):
            raise RuntimeError("peaks probe library not built: %s" % path)
        lib = ct.CDLL(path)
        for name in ("sasb200_probe_fp64_fma", "sasb200_probe_fp32_fma",
                     "sasb200_probe_mufu_sin"):
            fn = getattr(lib, name)
            fn.argtypes = [ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_void_p]
            fn.restype = ct.c_int32
        lib.sasb200_probe_threads_per_block.restype = ct.c_int32
        lib.sasb200_probe_chains.restype = ct.c_int32
        _LIB = lib
    return _LIB


def _measure(kind, iters=4096, blocks_per_sm=8, repeats=5):
    import torch
    lib = _lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    threads = lib.sasb200_probe_threads_per_block()
    chains = lib.sasb200_probe_chains()
    blocks = sms*blocks_per_sm
    dtype = torch.float64 if kind == "fp64" else torch.float32
    out = torch.empty(blocks*threads, dtype=dtype, device=dev)
    fn = {"fp64": lib.sasb200_probe_fp64_fma, "fp32": lib.sasb200_probe_fp32_fma,
          "mufu": lib.sasb200_probe_mufu_sin}[kind]
    stream = torch.cuda.current_stream(dev)
    for _ in range(2):
        if fn(out.data_ptr(), blocks, iters, stream.cuda_stream) != 0:
            raise RuntimeError("probe launch failed")
    best = float("inf")
    for _ in range(repeats):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        fn(out.data_ptr(), blocks, iters, stream.cuda_stream)
        stop.record(stream)
        stop.synchronize()
        best = min(best, start.elapsed_time(stop)*1e-3)
    ops = blocks*threads*chains*iters*(1 if kind == "mufu" else 2)
    return ops/best


def fp64_tflops():
    """Dense FP64 FMA throughput in TFLOP/s (2 flops per DFMA)."""
    return _measure("fp64")/1e12


def fp32_tflops():
    return _measure("fp32")/1e12


def mufu_tops():
    """__sinf evaluations per second, in T/s."""
    return _measure("mufu")/1e12


def measure_all():
    return dict(fp64_tflops=fp64_tflops(), fp32_tflops=fp32_tflops(),
                mufu_sin_tops=mufu_tops())
