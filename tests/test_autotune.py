"""
The autotuner's tile cache: a tuned tile is found again by key (CPU) and
used by later kernels of the same call shape through the public API (GPU).
"""

import numpy as np
import pytest


class _FakeLib:
    name = "cylinder"


class _FakeKernel:
    class meta:
        id = "cylinder"
    info = meta

    class q_input:
        nq = 65536

    lib = _FakeLib()
    device = 0


def test_cached_tile_lookup(tmp_path, monkeypatch):
    from sasmodels_b200 import autotune
    monkeypatch.setattr(autotune, "_FILE", str(tmp_path/"tune.json"))
    monkeypatch.setattr(autotune, "_CACHE", {})
    monkeypatch.setitem(autotune._NAMES, 0, "Fake GPU")
    k = _FakeKernel()
    assert autotune.cached_tile(k, "Iqxy", 490000) == 0
    autotune._CACHE[autotune._tile_key(k, "Iqxy", 490000)] = 0x000a0820
    autotune._save()
    # the same size class finds it, another variant or size class does not
    assert autotune.cached_tile(k, "Iqxy", 400000) == 0x000a0820
    assert autotune.cached_tile(k, "Imagnetic", 490000) == 0
    assert autotune.cached_tile(k, "Iqxy", 4900) == 0
    # a later process reads it back from the file
    monkeypatch.setattr(autotune, "_CACHE", {})
    assert autotune.cached_tile(k, "Iqxy", 490000) == 0x000a0820


@pytest.mark.gpu
def test_tuned_tile_reaches_public_calls(cuda, tmp_path, monkeypatch):
    import torch
    from sasmodels_b200 import autotune, load_model, workloads
    from sasmodels_b200.direct_model import make_call_args
    monkeypatch.setattr(autotune, "_FILE", str(tmp_path/"tune.json"))
    monkeypatch.setattr(autotune, "_CACHE", {})
    name, qv, pars = workloads.cylinder_2d(n=48, radius_n=5, length_n=5, theta_n=4, phi_n=4)
    model = load_model(name)
    details, values, magnetic = make_call_args(model.info, pars, qv)
    k1 = model.make_kernel(qv)
    dd, dv = k1.upload(details, values)
    variant = k1.variant(magnetic)
    tile = autotune.tune_kernel(k1, variant, dd, dv, details.num_eval, reps=1, budget_s=5.0)
    k1.stream.synchronize()
    seen = []
    k2 = model.make_kernel(qv)
    call = k2.lib.call

    def spy(*args):
        seen.append(args[12])
        return call(*args)
    monkeypatch.setattr(k2.lib, "call", spy)
    got = k2(details, values, 0.0, magnetic)
    assert seen == [tile]
    # the library's own tile gives the same sums to summation order
    k3 = model.make_kernel(qv)
    dd3, dv3 = k3.upload(details, values)
    with torch.cuda.stream(k3.stream):
        k3.launch(variant, dd3, dv3, 0, details.num_eval, 0.0, 0, tile=0)
    k3.stream.synchronize()
    raw2 = k2._result_dev.cpu().numpy()
    raw3 = k3._result_dev.cpu().numpy()
    np.testing.assert_allclose(raw2, raw3, rtol=1e-13, atol=0)
    assert np.all(np.isfinite(got))
