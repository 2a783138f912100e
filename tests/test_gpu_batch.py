"""
GPU tests of the batched population engine (sasmodels_b200.batch): every
set's raw sums and I(q) against the reference DLL, FP64 at the 1e-12 bar,
FP32c at 1e-5; graph capture/replay with new values; determinism.
"""

import numpy as np
import pytest

from helpers import (RTOL_FP64, compare_raw, full_size_population,
                     full_size_reference, load_info, marshal, normalise,
                     reference_raw)
from sasmodels_b200 import workloads
from sasmodels_b200.batch import Population

pytestmark = pytest.mark.gpu


def _pop(model, n, seed=1, max_pd_n=6):
    sets = [(q, p) for name, q, p in workloads.population(n_sets=2*n, seed=seed,
                                                          max_pd_n=max_pd_n)
            if name == model]
    return sets[:n]


@pytest.mark.parametrize("model", ["ellipsoid", "core_shell_cylinder"])
@pytest.mark.parametrize("form, rtol", [("double", RTOL_FP64), ("float32c", 1e-5)])
def test_batch_against_reference(cuda, model, form, rtol):
    sets = _pop(model, 10)
    pop = Population(model, sets, form=form, items_per_warp=64)
    pop.run()
    raws, iqs = pop.raw(), pop.iq()
    info = load_info(model)
    for (q, pars), raw, iq in zip(sets, raws, iqs):
        ref = reference_raw(model, info, [q], pars, threads=4)
        worst, f2rel = compare_raw(raw, ref, 2, len(q), rtol)
        assert worst <= 1.0, (model, form, worst, f2rel)
        _, values, _ = marshal(info, pars, [q])
        I_ref = normalise(ref, 2, len(q), values)["I"]
        np.testing.assert_allclose(iq, I_ref, rtol=max(rtol, 1e-13), atol=0)


def test_batch_graph_replay_and_update(cuda):
    model = "ellipsoid"
    sets = _pop(model, 8, seed=3)
    pop = Population(model, sets, form="float32c")
    pop.capture()
    pop.replay()
    first = [a.copy() for a in pop.iq()]
    # new values, same q and dispersity sizes
    new_pars = []
    for q, p in sets:
        p2 = dict(p)
        p2["sld"] = p["sld"] + 0.5
        p2["radius_equatorial"] = p["radius_equatorial"]*1.1
        new_pars.append(p2)
    pop.update(new_pars)
    pop.replay()
    after = pop.iq()
    fresh = Population(model, [(q, p) for (q, _), p in zip(sets, new_pars)], form="float32c")
    fresh.run()
    for a, b, c in zip(after, fresh.iq(), first):
        np.testing.assert_array_equal(a, b)
        assert not np.array_equal(a, c)


def test_batch_deterministic_and_tile_independent(cuda):
    model = "core_shell_cylinder"
    sets = _pop(model, 6, seed=5)
    a = Population(model, sets, form="float32c", items_per_warp=2)
    a.run()
    ra = a.raw()
    a.run()
    rb = a.raw()
    for x, y in zip(ra, rb):
        np.testing.assert_array_equal(x, y)
    # a different item split and block shape changes summation order only
    b = Population(model, sets, form="float32c", items_per_warp=256, warps=4)
    b.run()
    for x, y, (q, _) in zip(ra, b.raw(), sets):
        worst, _ = compare_raw(y, x, 2, len(q), 1e-12)
        assert worst <= 1.0


def test_batch_rejects_changed_structure(cuda):
    model = "ellipsoid"
    sets = _pop(model, 3, seed=7)
    pop = Population(model, sets)
    bad = [dict(p) for _, p in sets]
    key = [k for k in bad[0] if k.endswith("_pd_n")][0]
    bad[0][key] = bad[0][key] + 1
    with pytest.raises(ValueError):
        pop.update(bad)


def _line_sets(model, n, seed):
    rng = np.random.default_rng(seed)
    base = dict(workloads.population(n_sets=8, seed=seed, max_pd_n=5)[0 if model == "ellipsoid"
                                                                        else 1][2])
    sets = []
    for k in range(n):
        q = np.sort(rng.uniform(1e-3, 0.5, int(rng.integers(20, 200))))
        pars = {key: v for key, v in base.items() if not key.startswith("theta")
                and not key.startswith("phi")}
        pars["theta"] = 90.0 if k == 0 else float(rng.uniform(0, 180))
        pars["phi"] = 0.0 if k == 0 else float(rng.uniform(0, 360))
        sets.append((q, pars))
    return sets


@pytest.mark.parametrize("model", ["cylinder", "ellipsoid", "core_shell_cylinder"])
@pytest.mark.parametrize("form, rtol", [("double", RTOL_FP64), ("float32c", 1e-5)])
def test_line_form_against_reference_2d(cuda, model, form, rtol):
    """The line form equals the reference's 2D kernel at q vectors (q, 0)."""
    if model == "cylinder":
        sets = []
        rng = np.random.default_rng(5)
        for k in range(6):
            q = np.sort(rng.uniform(1e-3, 0.5, int(rng.integers(20, 200))))
            sets.append((q, dict(radius=float(rng.uniform(10, 300)),
                                 length=float(rng.uniform(20, 3000)),
                                 radius_pd=0.1*k/5, radius_pd_n=7,
                                 length_pd=0.2*k/5, length_pd_n=9, sld=3.0, sld_solvent=0.0,
                                 theta=90.0 if k < 2 else float(rng.uniform(0, 180)),
                                 phi=0.0 if k < 2 else float(rng.uniform(0, 360)))))
    else:
        sets = _line_sets(model, 5, 7)
    pop = Population(model, sets, form=form, line=True, items_per_warp=16)
    pop.run()
    info = load_info(model)
    for (q, pars), raw, iq in zip(sets, pop.raw(), pop.iq()):
        ref = reference_raw(model, info, [q, np.zeros_like(q)], pars, threads=4)
        nq = len(q)
        ours = np.concatenate([raw[0:2*nq:2], raw[2*nq:]])
        worst, f2rel = compare_raw(ours, ref, 1, nq, rtol)
        assert worst <= 1.0, (model, form, pars, worst, f2rel)


def test_batch_ragged_sets(cuda):
    """Sets of 1, 31, 32, 33 and 70 q points and a monodisperse set (mesh of
    one) in one population, against the DLL."""
    rng = np.random.default_rng(8)
    sets = []
    for nq, pd_n in [(1, 5), (31, 1), (32, 7), (33, 0), (70, 3)]:
        q = np.sort(rng.uniform(1e-3, 0.5, nq))
        sets.append((q, dict(radius_polar=float(rng.uniform(20, 200)),
                             radius_equatorial=float(rng.uniform(20, 200)),
                             radius_polar_pd=0.1, radius_polar_pd_n=pd_n)))
    pop = Population("ellipsoid", sets, form="double")
    pop.run()
    info = load_info("ellipsoid")
    for (q, pars), raw in zip(sets, pop.raw()):
        ref = reference_raw("ellipsoid", info, [q], pars)
        worst, f2rel = compare_raw(raw, ref, 2, len(q), RTOL_FP64)
        assert worst <= 1.0, (len(q), worst, f2rel)


@pytest.mark.parametrize("form, rtol", [("double", RTOL_FP64), ("float32c", 1e-5)])
def test_batch_full_size_against_reference(cuda, form, rtol):
    """The batched engine on population members at full size (dispersity
    meshes up to 287,430 points, the 500- and 5000-point Gauss rules), FP64
    at the 1e-12 bar and FP32c at 1e-5, raw sums and I(q) against the
    reference DLL."""
    by = {}
    for k, name, q, pars in full_size_population():
        by.setdefault(name, []).append((k, q, pars))
    for name, members in by.items():
        info = load_info(name)
        pop = Population(name, [(q, p) for _, q, p in members], form=form)
        pop.run()
        for (k, q, pars), raw, iq in zip(members, pop.raw(), pop.iq()):
            ref = full_size_reference(k, name, q, pars)
            worst, f2rel = compare_raw(raw, ref, 2, len(q), rtol)
            assert worst <= 1.0, (name, k, form, worst, f2rel)
            _, values, _ = marshal(info, pars, [q])
            I_ref = normalise(ref, 2, len(q), values)["I"]
            np.testing.assert_allclose(iq, I_ref, rtol=max(rtol, 1e-13), atol=0)
