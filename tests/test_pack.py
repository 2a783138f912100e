"""
Device-side marshaling of populations (csrc/pack.cu, pack.column_args,
batch.Population.from_columns): the column table and its CPU restatement
(oracle/pack_ref.py) against make_call_args on CPU, the device expansion
against the restatement and the set-by-set population on the GPU.
"""

import numpy as np
import pytest

from oracle import pack_ref

MODELS = ["cylinder", "ellipsoid", "core_shell_cylinder", "sphere", "core_shell_sphere"]


KINDS = ["gaussian", "lognormal", "schulz", "uniform", "rectangle", "boltzmann"]


def _columns(info, n, seed, clip=True, other_types=True, magnetic=False):
    """A random population as columns: values per set, dispersity widths,
    point counts and (with other_types) every distribution per set; with
    clip, widths that push points past a parameter limit; with magnetic,
    magnetic moments on some sets."""
    rng = np.random.default_rng(seed)
    cols = {}
    for p in info.parameters.kernel_parameters:
        if p.type == "sld":
            cols[p.name] = rng.uniform(-1, 7, n)
        elif p.polydisperse and p.type != "orientation":
            cols[p.name] = np.exp(rng.uniform(np.log(10), np.log(500), n))
        elif p.type == "orientation":
            cols[p.name] = rng.uniform(0, 90, n)
    for p in info.parameters.kernel_parameters:
        if not p.polydisperse:
            continue
        width = rng.uniform(0.0, 0.35, n)
        width[rng.uniform(size=n) < 0.2] = 0.0
        cols[p.name + "_pd"] = width if p.type != "orientation" else rng.uniform(0, 15, n)
        cols[p.name + "_pd_n"] = rng.choice([0, 1, 5, 35], n, p=[0.3, 0.04, 0.3, 0.36])
        if other_types and p.type != "orientation":
            cols[p.name + "_pd_type"] = np.array([KINDS[(i + len(p.name)) % len(KINDS)]
                                                  for i in range(n)], dtype=object)
    if clip:
        first = [p.name for p in info.parameters.kernel_parameters
                 if p.polydisperse and p.type != "orientation"][0]
        cols[first + "_pd"][::13] = 0.5
        cols[first + "_pd_n"][::13] = 9
    if magnetic:
        for p in info.parameters.kernel_parameters:
            if p.type == "sld":
                m0 = rng.uniform(0, 3, n)
                m0[::3] = 0.0
                cols[p.name + "_M0"] = m0
                cols[p.name + "_mtheta"] = rng.uniform(0, 180, n)
                cols[p.name + "_mphi"] = rng.uniform(0, 360, n)
        cols["up_frac_i"] = 0.9
        cols["up_frac_f"] = 0.8
    cols["scale"] = 1.0
    return cols


def _row(cols, s):
    out = {}
    for k, v in cols.items():
        v = np.asarray(v)
        v = v[()] if v.ndim == 0 else v[s]
        out[k] = v.item() if hasattr(v, "item") else v
    return out


def _check_values(got, want, nvalues, length, nmag=0, kinds=()):
    """Scalars and mesh points equal; weights to the ulps exp/log/lgamma may
    differ by (the schulz exponent z log z - ... cancels to ~1e-12 of its
    terms); magnetic components to the ulps sin/cos may differ by; zero
    padding."""
    a = nvalues + length
    b = nvalues + 2*length
    m = nvalues - 3*nmag
    assert got.shape == want.shape
    np.testing.assert_array_equal(got[:m], want[:m])
    np.testing.assert_allclose(got[m:nvalues], want[m:nvalues], rtol=2e-15,
                               atol=2e-15*np.max(np.abs(want[m:nvalues]), initial=0.0))
    np.testing.assert_array_equal(got[nvalues:a], want[nvalues:a])
    wtol = 1e-11 if "schulz" in kinds else 4e-15
    np.testing.assert_allclose(got[a:b], want[a:b], rtol=wtol, atol=0)
    np.testing.assert_array_equal(got[b:], want[b:])


def _kinds(cols, s):
    return [str(np.asarray(v)[s] if np.asarray(v).ndim else v)
            for k, v in cols.items() if k.endswith("_pd_type")]


def test_pairwise_sum_order_is_numpys():
    rng = np.random.default_rng(1)
    for n in list(range(1, 40)) + [127, 128, 129, 255, 256, 257, 600, 1031]:
        a = np.exp(-rng.uniform(0, 5, n)**2)
        assert pack_ref.pairwise_sum(a) == np.sum(a), n


@pytest.mark.parametrize("name", MODELS)
@pytest.mark.parametrize("dim", ["1d", "2d"])
def test_column_table_matches_make_call_args(name, dim):
    """Every set of a column table has make_call_args's details and values:
    bit for bit where the host marshals it, and through the restatement of
    the device expansion (weights within 2 ulp: only exp may differ)."""
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    from sasmodels_b200.pack import column_args
    info = load_model_info(name)
    n = 120
    cols = _columns(info, n, 7, magnetic=dim == "2d")
    ca = column_args(info, n, cols, dim)
    vals = pack_ref.expand(ca)
    q = [np.zeros(1)] if dim == "1d" else [np.zeros(1), np.zeros(1)]
    off = 0
    assert ca["host_values"], "the population exercises the host path"
    assert len(ca["host_values"]) < n//2       # one-point meshes go to the host
    kinds_on_device = set()
    for s in range(n):
        d0, v0, mag = make_call_args(info, _row(cols, s), q)
        np.testing.assert_array_equal(ca["det"][s], d0.buffer)
        assert ca["num_eval"][s] == d0.num_eval
        assert ca["val_sizes"][s] == v0.size
        assert bool(ca["magnetic"][s]) == mag
        got = vals[off:off + v0.size]
        off += v0.size
        if s in ca["host_values"]:
            assert np.array_equal(got, v0)
        else:
            kinds_on_device.update(pack_ref.KINDS[c] for c, m in zip(ca["kinds"][s],
                                                                     ca["npts"][s]) if m > 0)
            _check_values(got, v0, info.parameters.nvalues, int(d0.num_weights),
                          info.parameters.nmagnetic if mag else 0, _kinds(cols, s))
    assert kinds_on_device == set(pack_ref.KINDS)


def _magnetic_population(n, seed=0):
    """core_shell_sphere sets shaped like the magnetic headline: lognormal
    radius (pd 0.2, 51 points), gaussian thickness (pd 0.1, 21 points), the
    three slds' moments M0 ~ U[0,3], mtheta ~ U[0,180], mphi ~ U[0,360]."""
    rng = np.random.default_rng(seed)
    cols = dict(radius=rng.uniform(40, 80, n), radius_pd=0.2, radius_pd_n=51,
                radius_pd_type="lognormal", thickness=rng.uniform(5, 15, n),
                thickness_pd=0.1, thickness_pd_n=21, sld_core=1.0, sld_shell=2.0,
                sld_solvent=3.0, up_frac_i=0.9, up_frac_f=0.8, up_theta=90.0, up_phi=45.0)
    for sld in ("sld_core", "sld_shell", "sld_solvent"):
        cols[sld + "_M0"] = rng.uniform(0, 3, n)
        cols[sld + "_mtheta"] = rng.uniform(0, 180, n)
        cols[sld + "_mphi"] = rng.uniform(0, 360, n)
    return cols


def test_magnetic_lognormal_population_packs_without_host():
    """A population shaped like the magnetic headline is described entirely
    by the device table: no set is marshaled by make_call_args, and the
    restated expansion equals make_call_args's values."""
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    from sasmodels_b200.pack import column_args
    info = load_model_info("core_shell_sphere")
    n = 24
    cols = _magnetic_population(n)
    ca = column_args(info, n, cols, "2d")
    assert not ca["host_values"]
    assert ca["magnetic"].all()
    vals = pack_ref.expand(ca)
    off = 0
    q = [np.zeros(1), np.zeros(1)]
    for s in range(n):
        d0, v0, mag = make_call_args(info, _row(cols, s), q)
        assert mag
        np.testing.assert_array_equal(ca["det"][s], d0.buffer)
        _check_values(vals[off:off + v0.size], v0, info.parameters.nvalues,
                      int(d0.num_weights), info.parameters.nmagnetic, ["lognormal"])
        off += v0.size


def test_column_args_rejects_bad_columns():
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.pack import column_args
    info = load_model_info("sphere")
    with pytest.raises(TypeError, match="Unused"):
        column_args(info, 3, dict(radius=1.0, bogus=2.0))
    with pytest.raises(ValueError, match="shape"):
        column_args(info, 3, dict(radius=np.ones(4)))


@pytest.mark.parametrize("line", [False, True])
def test_host_pack_columns_layout_equals_sets(line):
    """A column population has the set-by-set population's descriptors,
    details and work items."""
    from sasmodels_b200.batch import host_pack, host_pack_columns
    from sasmodels_b200.core import load_model_info
    info = load_model_info("cylinder")
    n = 40
    cols = _columns(info, n, 3, other_types=False)
    if line:
        for k in ("theta_pd", "theta_pd_n", "phi_pd", "phi_pd_n"):
            cols.pop(k)
    rng = np.random.default_rng(4)
    qs = [np.geomspace(1e-3, 0.5, int(m)) for m in rng.integers(10, 300, n)]
    a = host_pack("cylinder", info, [(q, _row(cols, s)) for s, q in enumerate(qs)], line)
    b = host_pack_columns("cylinder", info, qs, cols, line)
    for key in ("desc", "q", "det", "items", "tile_off", "tile_items"):
        np.testing.assert_array_equal(a[key], b[key])
    for key in ("nq", "num_eval", "val_sizes", "pd_shape"):
        assert list(a[key]) == list(b[key]), key
    assert (a["n_tiles"], a["n_items"]) == (b["n_tiles"], b["n_items"])


def _gpu_population(model, n, seed, line=False):
    from sasmodels_b200.core import load_model_info
    info = load_model_info(model)
    cols = _columns(info, n, seed, other_types=False)
    if line:
        for p in info.parameters.kernel_parameters:
            if p.type == "orientation":
                cols.pop(p.name + "_pd", None)
                cols.pop(p.name + "_pd_n", None)
    rng = np.random.default_rng(seed + 1)
    qs = [np.geomspace(1e-3, 0.5, int(m)) for m in rng.integers(20, 400, n)]
    return info, cols, qs


@pytest.mark.gpu
@pytest.mark.parametrize("model, line", [("cylinder", False), ("ellipsoid", False),
                                         ("core_shell_cylinder", False), ("cylinder", True)])
def test_device_pack_matches_oracle_and_sets(cuda, model, line):
    """The values the device expands equal the restatement (weights within
    2 ulp), and I(q) equals the set-by-set population's to 1e-12."""
    from sasmodels_b200.batch import Population
    info, cols, qs = _gpu_population(model, 150, 11, line)
    pop = Population.from_columns(model, qs, cols, form="double", line=line)
    vals = pop.d_val.cpu().numpy()
    want = pack_ref.expand(pop.columns)
    off = 0
    for s in range(pop.n_sets):
        size = int(pop.columns["val_sizes"][s])
        length = int(pop.columns["lengths"][s].sum())
        if s in pop.columns["host_values"]:
            assert np.array_equal(vals[off:off + size], want[off:off + size])
        else:
            _check_values(vals[off:off + size], want[off:off + size],
                          info.parameters.nvalues, length)
        off += size
    pop.run()
    got = pop.iq()
    ref = Population(model, [(q, _row(cols, s)) for s, q in enumerate(qs)], form="double",
                     line=line)
    ref.run()
    for a, b in zip(got, ref.iq()):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["ellipsoid", "core_shell_cylinder"])
def test_device_pack_every_distribution(cuda, model):
    """Sets with every distribution of the plugin API and clipped meshes,
    packed on the device: values against the restatement, and the batched
    FP64 I(q) against the set-by-set (host-marshaled) population.  Schulz
    weights differ from the host's by up to ~1e-12 (its exponent cancels),
    so I(q) is held to 1e-11."""
    from sasmodels_b200.batch import Population
    from sasmodels_b200.core import load_model_info
    info = load_model_info(model)
    n = 90
    cols = _columns(info, n, 17)
    rng = np.random.default_rng(18)
    qs = [np.geomspace(1e-3, 0.5, int(m)) for m in rng.integers(20, 200, n)]
    pop = Population.from_columns(model, qs, cols, form="double")
    assert len(pop.columns["host_values"]) < n//2
    vals = pop.d_val.cpu().numpy()
    want = pack_ref.expand(pop.columns)
    off = 0
    for s in range(n):
        size = int(pop.columns["val_sizes"][s])
        length = int(pop.columns["lengths"][s].sum())
        if s in pop.columns["host_values"]:
            assert np.array_equal(vals[off:off + size], want[off:off + size])
        else:
            _check_values(vals[off:off + size], want[off:off + size],
                          info.parameters.nvalues, length, 0, _kinds(cols, s))
        off += size
    pop.run()
    ref = Population(model, [(q, _row(cols, s)) for s, q in enumerate(qs)], form="double")
    ref.run()
    for a, b in zip(pop.iq(), ref.iq()):
        np.testing.assert_allclose(a, b, rtol=1e-11, atol=0)


@pytest.mark.gpu
def test_device_pack_magnetic_drives_plain_kernel(cuda):
    """Magnetic headline-shaped sets packed on the device (lognormal and
    gaussian meshes, moments converted on the GPU) feed the plain Imagnetic
    kernel straight from device memory: I(q) within 1e-12 of the same call
    with host-marshaled values."""
    import torch
    from sasmodels_b200 import load_model
    from sasmodels_b200.batch import _Packer
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.pack import column_args
    from helpers import compare_raw, marshal
    info = load_model_info("core_shell_sphere")
    n = 6
    cols = _magnetic_population(n, seed=3)
    ca = column_args(info, n, cols, "2d")
    assert not ca["host_values"]
    model = load_model("core_shell_sphere")
    x = np.linspace(-0.1, 0.1, 24)
    qx, qy = [a.ravel() for a in np.meshgrid(x, x)]
    kernel = model.make_kernel([qx, qy])
    stream = kernel.stream
    d_val = torch.empty(int(ca["val_sizes"].sum()), dtype=torch.float64, device=kernel.device)
    packer = _Packer(ca, kernel.device, stream)
    packer.load(ca)
    packer.enqueue(d_val)
    stream.synchronize()
    off = 0
    for s in range(n):
        size = int(ca["val_sizes"][s])
        details, values, magnetic = marshal(info, _row(cols, s), [qx, qy])
        assert magnetic
        dev_d, _ = kernel.upload(details, values)
        nq = kernel.q_input.nq
        with torch.cuda.stream(stream):
            a = kernel.launch("Imagnetic", dev_d, d_val[off:off + size], 0,
                              details.num_eval, 0.0, 0).clone()
        kernel._call_kernel(details, values, 0.0, True, 0)
        stream.synchronize()
        b = kernel._result_dev.clone()
        worst, f2rel = compare_raw(a.cpu().numpy()[:nq + 4], b.cpu().numpy()[:nq + 4],
                                   1, nq, 1e-12)
        assert worst <= 1.0, (s, worst, f2rel)
        off += size


@pytest.mark.gpu
def test_update_columns_replays_in_graph(cuda):
    """A captured column population re-expanded from new columns by graph
    replay holds, bit for bit, the values of a fresh population of the new
    columns, and its I(q) (whose work items were cut for the old sizes)
    agrees to summation order."""
    import torch
    from sasmodels_b200.batch import Population
    info, cols, qs = _gpu_population("ellipsoid", 120, 21)
    pop = Population.from_columns("ellipsoid", qs, cols)
    pop.capture()
    new = dict(cols)
    rng = np.random.default_rng(5)
    for k in ("radius_polar", "radius_equatorial"):
        new[k] = cols[k]*rng.uniform(0.9, 1.1, len(qs))
    new["sld"] = rng.uniform(-1, 7, len(qs))
    pop.update_columns(new)
    pop.replay()
    got = pop.iq()
    fresh = Population.from_columns("ellipsoid", qs, new)
    fresh.run()
    assert torch.equal(pop.d_val, fresh.d_val)
    for a, b in zip(got, fresh.iq()):
        np.testing.assert_allclose(a, b, rtol=1e-13, atol=0)
    changed = dict(new)
    changed["radius_polar_pd_n"] = np.where(np.asarray(new["radius_polar_pd_n"]) == 35, 5, 35)
    with pytest.raises(ValueError, match="structure"):
        pop.update_columns(changed)


@pytest.mark.parametrize("flag", [0, 1])
def test_surrogate_columns_equal_model_pars(flag):
    """The surrogate's plain evaluations marshal the same sets as columns
    (model_columns) as set by set (model_pars)."""
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    from sasmodels_b200.pack import column_args
    from sasmodels_b200.surrogate import model_columns, model_pars, sample_sets
    info = load_model_info("cylinder")
    sets = sample_sets(60, np.random.default_rng(9))
    sets["rpd"][::5] = 0.0
    sets["lpd"][::7] = 0.0
    idx = np.arange(60)
    dim = "1d" if flag else "2d"
    ca = column_args(info, 60, model_columns(sets, idx, flag), dim)
    vals = pack_ref.expand(ca)
    q = [np.zeros(1)] if flag else [np.zeros(1), np.zeros(1)]
    off = 0
    for s in idx:
        pars = model_pars(sets["radius"][s], sets["length"][s], sets["rpd"][s], sets["lpd"][s],
                          flag)
        d0, v0, _ = make_call_args(info, pars, q)
        np.testing.assert_array_equal(ca["det"][s], d0.buffer)
        _check_values(vals[off:off + v0.size], v0, info.parameters.nvalues,
                      int(d0.num_weights))
        off += v0.size


def test_columns_from_sets_round_trip():
    """Columns gathered from parameter dicts marshal every set as the dict
    itself does (missing dispersity fields take their defaults)."""
    from sasmodels_b200 import workloads
    from sasmodels_b200.core import load_model_info
    from sasmodels_b200.direct_model import make_call_args
    from sasmodels_b200.pack import column_args, columns_from_sets
    pop = [(q, p) for name, q, p in workloads.population(n_sets=200, seed=3)
           if name == "core_shell_cylinder"]
    info = load_model_info("core_shell_cylinder")
    pars = [p for _, p in pop]
    ca = column_args(info, len(pars), columns_from_sets(info, pars))
    vals = pack_ref.expand(ca)
    off = 0
    for s, p in enumerate(pars):
        d0, v0, _ = make_call_args(info, p, [np.zeros(1)])
        np.testing.assert_array_equal(ca["det"][s], d0.buffer)
        _check_values(vals[off:off + v0.size], v0, info.parameters.nvalues,
                      int(d0.num_weights))
        off += v0.size
