"""
Project autotuner: picks launch shapes by timing candidates on the device.

* :func:`tune_kernel` chooses the ``iq_main`` tile (lanes per q, warps per
  block, mesh splits) for one kernel call shape;
* :func:`tune_population` chooses the batched engine's warps per block and
  items per warp for a population.

Choices are cached in memory and in a JSON file keyed by device name, model,
variant and a size class, so a process tunes each shape once
(``SASB200_TUNE_CACHE`` overrides the file, empty disables it).
"""

import json
import os
import time

import numpy as np

_CACHE = {}
_FILE = os.environ.get("SASB200_TUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "sasmodels_b200",
                                    "autotune.json"))


def _load():
    if _CACHE or not _FILE:
        return
    try:
        with open(_FILE) as fid:
            _CACHE.update(json.load(fid))
    except (OSError, ValueError):
        pass


def _save():
    if not _FILE:
        return
    try:
        os.makedirs(os.path.dirname(_FILE), exist_ok=True)
        # one writer per process (one process per GPU): write aside, then
        # rename, so readers never see a partial file
        tmp = "%s.%d.tmp" % (_FILE, os.getpid())
        with open(tmp, "w") as fid:
            json.dump(_CACHE, fid, indent=0)
        os.replace(tmp, _FILE)
    except OSError:
        pass


def _size_class(n):
    return int(np.ceil(np.log2(max(n, 1))))


_NAMES = {}


def _device_name(device):
    import torch
    index = torch.device(device).index if not isinstance(device, int) else device
    if index is None:
        index = torch.cuda.current_device()
    if index not in _NAMES:
        _NAMES[index] = torch.cuda.get_device_name(index)
    return _NAMES[index]


def _tile_key(kernel, variant, n_mesh):
    return "|".join(["tile", _device_name(kernel.device), kernel.meta.id, kernel.lib.name,
                     variant, str(_size_class(kernel.q_input.nq)), str(_size_class(n_mesh))])


def cached_tile(kernel, variant, n_mesh):
    """The tile code `tune_kernel` chose for this call shape (this device,
    model, variant and size class), in this process or an earlier one whose
    cache file is shared; 0 (the library's choice) when there is none."""
    _load()
    return int(_CACHE.get(_tile_key(kernel, variant, n_mesh), 0))


def _time_stream(fn, stream, reps=2):
    import torch
    fn()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(reps):
        fn()
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop)/reps


def tile_candidates(lib, nq, n_mesh, sms=148):
    """Instantiated (lanes, warps) shapes x a few mesh-split counts."""
    out = []
    nseg = max(1, (n_mesh + 127)//128)
    for code in lib.tile_shapes():
        lq, warps = code & 0xff, (code >> 8) & 0xff
        qtiles = max(1, (nq + lq - 1)//lq)
        for blocks_per_sm in (8, 32, 128, 512):
            splits = int(min(nseg, max(1, np.ceil(sms*blocks_per_sm/qtiles)), 128))
            out.append((splits << 16) | (warps << 8) | lq)
    return sorted(set(out))


def tune_kernel(kernel, variant, details_dev, values_dev, n_mesh, reps=2, budget_s=20.0):
    """Set ``kernel.tile`` to the fastest tile code for this call shape and
    return it."""
    import torch
    _load()
    key = _tile_key(kernel, variant, n_mesh)
    if key in _CACHE:
        kernel.tile = int(_CACHE[key])
        return kernel.tile
    sms = torch.cuda.get_device_properties(kernel.device).multi_processor_count
    best, best_t = 0, float("inf")
    t_start = time.perf_counter()
    kernel._tuning = True          # code 0 is the library's own choice here
    try:
        for code in [0] + tile_candidates(kernel.lib, kernel.q_input.nq, n_mesh, sms):
            kernel.tile = code

            def call():
                kernel.launch(variant, details_dev, values_dev, 0, n_mesh, 0.0, 0)
            with torch.cuda.stream(kernel.stream):
                t = _time_stream(call, kernel.stream, reps)
            if t < best_t:
                best, best_t = code, t
            if time.perf_counter() - t_start > budget_s:
                break
    finally:
        kernel._tuning = False
    kernel.tile = best
    _CACHE[key] = best
    _save()
    return best


def tune_population(model, sets, form="float32c", subsample=48, reps=1,
                    candidates=((8, 8), (4, 8), (8, 32), (4, 32), (8, 2))):
    """(warps, items_per_warp) with the least time on an evenly spaced
    subsample of *sets*."""
    import torch
    from .batch import Population
    _load()
    key = "|".join(["pop", _device_name(torch.cuda.current_device()), model, form,
                    str(_size_class(len(sets)))])
    if key in _CACHE:
        return tuple(_CACHE[key])
    idx = np.linspace(0, len(sets) - 1, min(subsample, len(sets))).astype(int)
    sample = [sets[i] for i in sorted(set(idx))]
    best, best_t = candidates[0], float("inf")
    for warps, ipw in candidates:
        pop = Population(model, sample, form=form, warps=warps, items_per_warp=ipw)
        t = _time_stream(pop.run, pop.stream, reps)
        if t < best_t:
            best, best_t = (warps, ipw), t
    _CACHE[key] = list(best)
    _save()
    return best
