"""
CPU tests: the host-side mirror of the reference call path, the oracle pinned
against the reference's golden vectors, and the C-ABI libraries' exports.
No GPU is touched here.
"""

import ctypes as ct
import os
import re

import numpy as np
import pytest

from helpers import (MODELS, golden, interleave, is_near, load_info, marshal,
                     normalise, nout_of, variant)
from sasmodels_b200 import _abi, weights
from sasmodels_b200.generate import device_source, find_xy_mode

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


@pytest.mark.parametrize("name", MODELS)
def test_marshal_matches_reference(name):
    """get_mesh + make_kernel_args reproduce the reference's packed arrays."""
    info = load_info(name)
    for case in golden(name)["marshal"]:
        details, values, magnetic = marshal(info, case["pars"], case["q"])
        np.testing.assert_array_equal(details.buffer, case["details"])
        np.testing.assert_array_equal(values, np.array(case["values"]))
        assert magnetic == case["magnetic"]


@pytest.mark.parametrize("name", MODELS)
def test_oracle_reproduces_reference_dll(name):
    """oracle/_ref gives bitwise the raw vectors the reference's own
    DllKernel produced on the same inputs."""
    from oracle import refdll
    info = load_info(name)
    dll = refdll.load(name)
    for case in golden(name)["dll"]:
        nout = nout_of(info, case["dim"])
        raw = dll.call(variant(case["dim"], case["magnetic"]),
                       interleave(case["q"]), case["details"],
                       np.array(case["values"]), nout)
        np.testing.assert_array_equal(raw, np.array(case["raw"]))


@pytest.mark.parametrize("name", MODELS)
def test_oracle_against_model_golden_tests(name):
    """The oracle meets each model's embedded test values at 5 significant
    digits (the reference harness rule, model_test.py:443-471)."""
    info = load_info(name)
    from helpers import reference_raw
    for case in golden(name)["tests"]:
        pars = dict(case["pars"])
        reff_mode = int(pars.pop("radius_effective_mode", 1 if case["kind"] == "Fq" else 0))
        raw = reference_raw(name, info, case["q"], pars, reff_mode=reff_mode)
        details, values, _ = marshal(info, pars, case["q"])
        nq = len(case["q"][0])
        out = normalise(raw, nout_of(info, case["dim"]), nq, values)
        if case["kind"] == "I":
            for t, a in zip(case["y"], out["I"]):
                assert is_near(t, a), (name, case, t, a)
        else:
            if out["F1"] is not None:
                for t, a in zip(case["F"], out["F1"]):
                    assert is_near(t, a), (name, "F", t, a)
            for t, a in zip(case["F2"], out["F2"]):
                assert is_near(t, a), (name, "F2", t, a)
            assert is_near(case["reff"], out["reff"])
            assert is_near(case["volume"], out["shell"])
            assert is_near(case["volume_ratio"], out["ratio"])


def test_weights_normalised_and_truncated():
    v, w = weights.get_weights("gaussian", 35, 0.1, 3, 50.0, (0, np.inf), True)
    assert len(v) == 35 and abs(w.sum() - 1) < 1e-15
    assert v.min() == pytest.approx(35.0) and v.max() == pytest.approx(65.0)
    # truncation at the lower limit
    v, w = weights.get_weights("gaussian", 35, 0.5, 3, 1.0, (0, np.inf), True)
    assert v.min() >= 0 and len(v) < 35
    # orientation jitter is absolute and centred on zero
    v, w = weights.get_weights("gaussian", 5, 10.0, 3, 60.0, (-180, 180), False)
    assert v[len(v)//2] == 0.0


def test_too_many_polydisperse_parameters():
    from sasmodels_b200.details import make_details
    info = load_info("sphere")
    with pytest.raises(ValueError):
        make_details(info, np.array([2, 2, 2]), np.array([0, 2, 4]), 6)


def test_device_source_lexer():
    code = """
// comment with double foo(
static double f(double x) { constant double *w = T; return x*w[0]; }
constant double T[2] = {1.0, 2.0};
constant double BIG[5000] = {1.0};
double g(double);
typedef struct { double a; } S;
#define X(a) (a)
double sas_3j1x_x(double q)
{
    if (q < 0) { return 1.0; }
    return q;
}
"""
    out = device_source(code)
    assert "__device__ static double f(double x) { const double *w" in out
    assert "__constant__ const double T[2]" in out
    assert "__device__ const double BIG[5000]" in out
    assert "__device__ double g(double);" in out
    assert "typedef struct { double a; } S;" in out
    assert "__device__ double sas_3j1x_x(double q)" in out
    assert "#define X(a) (a)" in out
    assert find_xy_mode(["double Iqac(double qab, double qc)"]) == "qac"
    assert find_xy_mode(["static double Iq(double q)"]) == "qa"


def _header_suffixes():
    text = open(os.path.join(ROOT, "include", "sasb200.h")).read()
    block = text[text.index("#define SASB200_DECLARE_MODEL"):]
    block = block[:block.index("SASB200_DECLARE_MODEL(sphere)")]
    return sorted(set(re.findall(r"sasb200_##M##_(\w+)\(", block)))


def test_header_declares_models():
    text = open(os.path.join(ROOT, "include", "sasb200.h")).read()
    for name in MODELS:
        assert "SASB200_DECLARE_MODEL(%s)" % name in text


@pytest.mark.parametrize("name", MODELS)
def test_library_exports_header_symbols(name):
    """Each built library loads without a GPU and exports every symbol the
    header declares for it."""
    path = _abi.library_path(name)
    assert os.path.exists(path), "library not built: %s" % path
    lib = ct.CDLL(path)
    for prefix in (name, name + "_f32c"):
        for suffix in _header_suffixes():
            getattr(lib, "sasb200_%s_%s" % (prefix, suffix))
    text = open(os.path.join(ROOT, "include", "sasb200.h")).read()
    assert "SASB200_DECLARE_BATCH(%s)" % name in text
    getattr(lib, "sasb200_%s_batch" % name)
    meta = _abi.load_metadata(name)
    assert meta["id"] == name


@pytest.mark.parametrize("name", MODELS)
def test_abi_host_queries(name):
    """Size and tile queries run on the host (no kernel launch)."""
    lib = _abi.load_library(name)
    shapes = lib.tile_shapes()
    assert len(shapes) >= 1 and all(s & 0xff in (1, 8, 32) for s in shapes)
    n = lib.workspace_bytes("Iq", 1000, 35)
    assert n >= 35*8 and n % 256 == 0
    assert lib.workspace_bytes("Iqxy", 65536, 490000, 0) > 490000*8
    tile = lib.default_tile("Iqxy", 1000, 35)
    assert (tile & 0xff) in (1, 8, 32)
    # 1D: one q per warp; large 2D: 32 neighbouring q per warp, many splits
    assert lib.default_tile("Iq", 1000, 1225) & 0xff == 1
    big = lib.default_tile("Iqxy", 65536, 490000)
    assert big & 0xff == 32 and 16 <= (big >> 16) <= 128


def test_abi_rejects_bad_arguments_without_gpu():
    """Argument checks happen before any CUDA call."""
    lib = _abi.load_library("sphere")
    with pytest.raises(RuntimeError, match="pd_start"):
        lib.call("Iq", 10, 5, 3, 1, 1, 1, 1, 0.0, 0, 1, 1 << 20, 0, None)
    with pytest.raises(RuntimeError, match="null"):
        lib.call("Iq", 10, 0, 3, None, 1, 1, 1, 0.0, 0, 1, 1 << 20, 0, None)
    with pytest.raises(RuntimeError, match="tile"):
        lib.call("Iq", 10, 0, 3, 1, 1, 1, 1, 0.0, 0, 1, 1 << 20, 0x10307, None)
    # a mesh range above the single-launch limit needs a workspace
    with pytest.raises(RuntimeError, match="workspace"):
        lib.call("Iq", 10, 0, 100000, 1, 1, 1, 1, 0.0, 0, 1, 16, 0, None)


def test_line_form_refuses_orientation_dispersion():
    from sasmodels_b200.batch import line_call_args
    from sasmodels_b200.core import load_model_info
    info = load_model_info("cylinder")
    q = np.linspace(0.01, 0.2, 5)
    details, values = line_call_args(info, dict(radius=20, radius_pd=0.1, radius_pd_n=5,
                                                theta=30, phi=10), q)
    assert details.num_eval == 5
    with pytest.raises(ValueError, match="orientation dispersion"):
        line_call_args(info, dict(radius=20, theta=30, theta_pd=5, theta_pd_n=3), q)


def test_gate_thresholds():
    """Per-tolerance thresholds keep the accepted points' violation rate
    at or below alpha, and grow with the tolerance."""
    from sasmodels_b200.surrogate import gate_thresholds
    rng = np.random.default_rng(0)
    err = np.exp(rng.normal(-6, 1.5, 200000))
    r = err*np.exp(rng.normal(0, 0.5, err.size))       # a noisy predictor
    tols = np.array([1e-3, 1e-2, 5e-2])
    th = gate_thresholds(r, err, tols, 1e-3)
    assert np.all(np.diff(th) >= 0)
    for tol, t in zip(tols, th):
        acc = r <= t
        assert acc.any()
        assert np.mean(err[acc] > tol) <= 1e-3 + 1e-12
    # a useless predictor accepts nothing at a tight tolerance
    assert gate_thresholds(np.ones(100), np.ones(100), [1e-3], 1e-3)[0] == 0.0


def test_error_envelope():
    from sasmodels_b200.surrogate import envelope
    err = np.array([0., 1., 0., 0., 0., 5., 0., 0.])
    sid = np.array([0, 0, 0, 0, 1, 1, 1, 1])
    # the maximum spreads two places each way, never across sets
    np.testing.assert_array_equal(envelope(err, sid, 2), [1., 1., 1., 1., 5., 5., 5., 5.])
    np.testing.assert_array_equal(envelope(err, sid, 0), err)


@pytest.mark.parametrize("name", ["cylinder", "ellipsoid", "core_shell_cylinder", "sphere",
                                  "core_shell_sphere"])
@pytest.mark.parametrize("dim", ["1d", "2d"])
def test_bulk_call_args_equal_single(name, dim):
    """Marshaling a population in one pass gives, set by set, the same
    details and values (bitwise) as make_call_args."""
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    from sasmodels_b200.pack import bulk_call_args
    info = load_model_info(name)
    rng = np.random.default_rng(7)
    vol = [p.name for p in info.parameters.kernel_parameters if p.polydisperse]
    orient = set(p.name for p in info.parameters.kernel_parameters if p.type == "orientation")
    pars_list = []
    for k in range(60):
        pars = {}
        for p in info.parameters.kernel_parameters:
            if p.type == "sld":
                pars[p.name] = float(rng.uniform(-1, 7))
            elif p.polydisperse and p.type != "orientation":
                pars[p.name] = float(np.exp(rng.uniform(np.log(10), np.log(500))))
        for p in vol:
            if rng.uniform() < 0.6:
                pars[p + "_pd"] = float(rng.uniform(0.0, 0.35)) if k % 7 else 0.0
                pars[p + "_pd_n"] = int(rng.choice([0, 1, 5, 35]))
                if k % 11 == 0 and p not in orient:
                    pars[p + "_pd_type"] = "lognormal"
        if k % 13 == 0:                 # wide enough to clip at zero
            pars[vol[0] + "_pd"] = 0.5
            pars[vol[0] + "_pd_n"] = 9
        pars_list.append(pars)
    q = [np.zeros(1)] if dim == "1d" else [np.zeros(1), np.zeros(1)]
    bulk = bulk_call_args(info, pars_list, dim)
    for pars, (d, v, m) in zip(pars_list, bulk):
        d0, v0, m0 = make_call_args(info, pars, q)
        np.testing.assert_array_equal(d.buffer, d0.buffer)
        assert v.dtype == v0.dtype and v.shape == v0.shape
        assert np.array_equal(v, v0), (name, pars)
        assert m == m0


def test_bulk_call_args_rejects_unknown():
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.pack import bulk_call_args
    with pytest.raises(TypeError, match="Unused"):
        bulk_call_args(load_model_info("sphere"), [dict(radius=1, bogus=2)])


@pytest.mark.parametrize("line", [False, True])
def test_host_pack_population(line):
    """Host packing of a population: every set's arrays equal the single-call
    marshaling, and the work items cover each (set, tile) mesh exactly once,
    in mesh order within the tile."""
    from sasmodels_b200.batch import host_pack
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    model = "cylinder" if line else "ellipsoid"
    info = load_model_info(model)
    rng = np.random.default_rng(3)
    sets = []
    for k in range(40):
        q = np.sort(rng.uniform(1e-3, 0.5, int(rng.integers(1, 300))))
        if line:
            pars = dict(radius=float(rng.uniform(10, 300)), length=float(rng.uniform(20, 3000)),
                        radius_pd=0.1, radius_pd_n=int(rng.choice([1, 5, 35])),
                        length_pd=0.05*(k % 3), length_pd_n=35, theta=90.0, phi=0.0)
        else:
            pars = dict(radius_polar=float(rng.uniform(10, 500)),
                        radius_equatorial=float(rng.uniform(10, 500)),
                        radius_polar_pd=0.2*(k % 2), radius_polar_pd_n=int(rng.integers(1, 20)))
        sets.append((q, pars))
    h = host_pack(model, info, sets, line=line, warps=8, items_per_warp=4, sms=8)
    items, off, lst = h["items"], h["tile_off"], h["tile_items"]
    for s, (q, pars) in enumerate(sets):
        d, v, _ = make_call_args(info, pars, [q, 0*q] if line else [q])
        nq_, qo, do, vo, ne, ro, io, to = h["desc"][s]
        assert nq_ == q.size and ne == d.num_eval
        np.testing.assert_array_equal(h["q"][qo:qo + nq_], q)
        np.testing.assert_array_equal(h["det"][do:do + d.buffer.size], d.buffer)
        assert np.array_equal(h["val"][vo:vo + v.size], v)
        for t in range((q.size + 31)//32):
            its = items[lst[off[to + t]:off[to + t + 1]]]
            assert np.all(its[:, 0] == s) and np.all(its[:, 1] == 32*t)
            assert its[0, 2] == 0 and its[-1, 3] == ne
            np.testing.assert_array_equal(its[1:, 2], its[:-1, 3])
    assert len(lst) == len(items) == len(set(lst.tolist()))


@pytest.mark.parametrize("lib_name", ["mlp", "peaks", "resolution", "pack"])
def test_support_libraries_export_header_symbols(lib_name):
    """libsasb200_{mlp,peaks,resolution,pack}.so load without a GPU and
    export every function their header (include/sasb200_mlp.h,
    include/sasb200_resolution.h, include/sasb200_pack.h) declares for
    them."""
    header = ("sasb200_%s.h" % lib_name if lib_name in ("resolution", "pack")
              else "sasb200_mlp.h")
    text = open(os.path.join(ROOT, "include", header)).read()
    names = sorted(set(re.findall(r"\b(sasb200_\w+)\(", text)))
    want = (names if lib_name in ("resolution", "pack") else
            [n for n in names if n.startswith("sasb200_probe") == (lib_name == "peaks")])
    assert want
    lib = ct.CDLL(os.path.join(_abi.LIB_DIR, "libsasb200_%s.so" % lib_name))
    for n in want:
        getattr(lib, n)


def test_device_locality_order_matches_host():
    """The Morton order computed with tensor operations (run here on the
    CPU; on the GPU in make_kernel) is the host function's permutation,
    ties included, and is a permutation."""
    import torch
    from sasmodels_b200.kernel import locality_order, locality_order_device
    rng = np.random.default_rng(9)
    for qx, qy in ((rng.uniform(-0.3, 0.5, 5000), rng.uniform(-0.1, 0.1, 5000)),
                   (np.repeat(np.linspace(-1, 1, 64), 64), np.tile(np.linspace(-1, 1, 64), 64)),
                   (np.full(100, 0.25), rng.uniform(0, 1, 100))):
        want = locality_order(qx, qy)
        got = locality_order_device(torch.as_tensor(qx), torch.as_tensor(qy)).numpy()
        np.testing.assert_array_equal(got, want)
