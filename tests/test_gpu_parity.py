"""
GPU parity: the sm_100a kernels through the C-ABI against the reference DLL
oracle (oracle/_ref) on identical packed inputs.

Bar (FP64 path): every F^2 slot and norm within rel 1e-12 of the DLL; every
<F> slot within 1e-12 of its Cauchy-Schwarz scale sqrt(sum w * sum w F^2)
(see helpers.compare_raw).  The embedded model tests are also checked at the
reference harness's 5 significant digits.
"""

import numpy as np
import pytest

from helpers import (FULL_SIZE_SETS, MODELS, RTOL_FP64, compare_raw,
                     full_size_population, full_size_reference, gauss_rule_counts,
                     golden, host_threads, interleave, is_near, load_info, marshal,
                     normalise, nout_of, reference_raw, variant)
from sasmodels_b200 import direct_model, load_model, workloads

pytestmark = pytest.mark.gpu


def gpu_raw(name, q_vectors, pars, cutoff=0.0, reff_mode=0, tile=0):
    model = load_model(name)
    kernel = model.make_kernel([np.asarray(v, 'd') for v in q_vectors])
    kernel.tile = tile
    details, values, magnetic = marshal(model.info, pars, q_vectors)
    kernel._call_kernel(details, values, cutoff, magnetic, reff_mode)
    nout = nout_of(model.info, kernel.dim)
    nq = kernel.q_input.nq
    raw = np.concatenate([kernel.result[:nout*nq], kernel.result[nout*nq:nout*nq+4]])
    return raw, nout, nq, values


def assert_parity(name, q_vectors, pars, cutoff=0.0, reff_mode=0, tile=0,
                  rtol=RTOL_FP64, threads=8):
    info = load_info(name)
    ours, nout, nq, values = gpu_raw(name, q_vectors, pars, cutoff, reff_mode, tile)
    ref = reference_raw(name, info, q_vectors, pars, cutoff, reff_mode,
                        threads=threads)
    worst, f2rel = compare_raw(ours, ref, nout, nq, rtol)
    assert worst <= 1.0, "%s: worst err %.3g x tol (max F^2 rel %.3g)" % (
        name, worst, f2rel)
    return ours, ref


@pytest.mark.parametrize("name", MODELS)
def test_golden_dll_cases(cuda, name):
    """Seeded 1D/2D/magnetic cases recorded from the reference DLL."""
    info = load_info(name)
    for case in golden(name)["dll"]:
        ours, nout, nq, values = gpu_raw(name, case["q"], case["pars"])
        np.testing.assert_array_equal(values, np.array(case["values"]))
        worst, f2rel = compare_raw(ours, np.array(case["raw"]), nout, nq)
        assert worst <= 1.0, (name, case["dim"], worst, f2rel)


@pytest.mark.parametrize("name", MODELS)
def test_model_golden_values(cuda, name):
    """Each model's embedded test values, through the drop-in API
    (direct_model.call_kernel / call_Fq on a B200Kernel)."""
    model = load_model(name)
    for case in golden(name)["tests"]:
        qv = [np.asarray(v, 'd') for v in case["q"]]
        kernel = model.make_kernel(qv)
        pars = dict(case["pars"])
        if case["kind"] == "I":
            out = direct_model.call_kernel(kernel, pars)
            for t, a in zip(case["y"], out):
                assert is_near(t, a), (name, case["pars"], t, a)
        else:
            F1, F2, reff, shell, ratio = direct_model.call_Fq(kernel, pars)
            if F1 is not None:
                for t, a in zip(case["F"], F1):
                    assert is_near(t, a), (name, "F", t, a)
            for t, a in zip(case["F2"], F2):
                assert is_near(t, a), (name, "F2", t, a)
            assert is_near(case["reff"], reff)
            assert is_near(case["volume"], shell)
            assert is_near(case["volume_ratio"], ratio)
        # and the same points at the FP64 bar against the live oracle
        pars.pop("radius_effective_mode", None)
        assert_parity(name, case["q"], pars, threads=1)


def test_sphere_config_full(cuda):
    """sphere 1D headline configuration at full size (1000 q x 35 mesh)."""
    name, qv, pars = workloads.sphere_1d()
    assert_parity(name, qv, pars)


def test_cylinder_2d_full_mesh_subgrid(cuda):
    """cylinder 2D oriented: full 490000-point mesh on an 8x8 q block of the
    256x256 grid."""
    name, qv, pars = workloads.cylinder_2d_subgrid(8)
    assert_parity(name, qv, pars)


@pytest.mark.parametrize("where", ["corner", "strided"])
def test_cylinder_2d_full_mesh_off_centre(cuda, where):
    """cylinder 2D oriented at the full 490000-point mesh away from the grid
    centre: the corner 8x8 block (|q| up to 0.42 1/A; 56 % of evaluations
    take the asymptotic J1 branch, x = qab*R > 5, models/lib/sas_J1.c) and a
    strided 16x16 sample of the whole grid (every 16th row and column; 21 %
    asymptotic, the branch mix of the full grid).  Here the cancellation in
    qab^2 = |q|^2 - qc^2 and the J1 large-argument form both run."""
    if where == "corner":
        name, qv, pars = workloads.cylinder_2d_subgrid(8, where="corner")
        least = 0.5
    else:
        name, qv, pars = workloads.cylinder_2d_strided(16)
        least = 0.15
    assert workloads.cylinder_j1_large_fraction(qv[0], qv[1], pars) > least
    assert_parity(name, qv, pars, threads=host_threads())


@pytest.mark.parametrize("k", list(FULL_SIZE_SETS))
def test_population_full_size(cuda, k):
    """Population members at full size (dispersity meshes up to
    67 x 59 x 68 points, the 500- and 5000-point Gauss rules) through the
    plain FP64 kernel against the reference DLL, on a q subsample of each
    set that keeps its smallest and largest q."""
    (_, name, q, pars), = [c for c in full_size_population() if c[0] == k]
    rules = gauss_rule_counts(name, q, pars)
    if k in (1747, 563):
        assert rules[5000] > 0, rules
    ours, nout, nq, values = gpu_raw(name, [q], pars)
    ref = full_size_reference(k, name, q, pars)
    worst, f2rel = compare_raw(ours, ref, nout, nq)
    assert worst <= 1.0, "%s set %d: worst err %.3g x tol (max F^2 rel %.3g)" % (
        name, k, worst, f2rel)


def test_magnetic_full_mesh_subgrid(cuda):
    """core_shell_sphere magnetic: full 1071-point mesh, 16x16 q block."""
    name, (qx, qy), pars = workloads.core_shell_sphere_magnetic(n=128)
    sub = np.arange(0, 128*128, 64)
    assert_parity(name, [qx[sub], qy[sub]], pars)


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_population_members(cuda, k):
    """Members of the fit population (ellipsoid / core_shell_cylinder 1D
    with adaptive quadrature), reduced mesh."""
    pop = workloads.population(n_sets=8, seed=1, max_pd_n=9)
    name, q, pars = pop[k]
    assert_parity(name, [q], pars)


@pytest.mark.parametrize("tile", [0x00010420, 0x00030408, 0x00020801, 0x00050808, 0x00010801])
def test_tile_shapes_agree(cuda, tile):
    """Every tile shape gives the oracle's answer (reduction order differs,
    the result must not)."""
    _, qv, pars = workloads.cylinder_2d(n=12, radius_n=7, length_n=5,
                                        theta_n=5, phi_n=4)
    assert_parity("cylinder", qv, pars, tile=tile)


def test_restart_matches_single_call(cuda):
    """pd_start/pd_stop restart: two calls over halves of the mesh give the
    single-call sums (kernel_iq.c:381-423 contract)."""
    import torch
    name, qv, pars = workloads.cylinder_2d(n=10, radius_n=5, length_n=5,
                                           theta_n=4, phi_n=3)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    n = details.num_eval
    with torch.cuda.stream(kernel.stream):
        full = kernel.launch("Iqxy", dev_d, dev_v, 0, n, 0.0, 0).clone()
        part = torch.zeros_like(full)
        kernel.launch("Iqxy", dev_d, dev_v, 0, n//3, 0.0, 0, result_dev=part)
        kernel.launch("Iqxy", dev_d, dev_v, n//3, n, 0.0, 0, result_dev=part)
    kernel.stream.synchronize()
    full = full.cpu().numpy()
    part = part.cpu().numpy()
    nq = kernel.q_input.nq
    worst, _ = compare_raw(part[:nq+4], full[:nq+4], 1, nq, 1e-13)
    assert worst <= 1.0


def test_cutoff_and_reff(cuda):
    """cutoff > 0 drops light mesh points; R_eff accumulated when asked."""
    name = "cylinder"
    q = np.logspace(-3, -0.5, 50)
    pars = dict(radius=30., radius_pd=0.2, radius_pd_n=25, length=200.,
                length_pd=0.3, length_pd_n=25)
    assert_parity(name, [q], pars, cutoff=1e-4, reff_mode=1)
    assert_parity(name, [q], pars, cutoff=0.0, reff_mode=7)


def test_deterministic(cuda):
    name, qv, pars = workloads.sphere_1d(nq=333)
    a, *_ = gpu_raw(name, qv, pars)
    b, *_ = gpu_raw(name, qv, pars)
    np.testing.assert_array_equal(a, b)


def test_edge_cases(cuda):
    """single q, monodisperse (mesh of one), q = 0 in the magnetic kernel,
    empty mesh range."""
    assert_parity("sphere", [np.array([0.05])], dict(radius=80.), threads=1)
    assert_parity("cylinder", [np.array([0.0, 1e-3]), np.array([0.0, 2e-3])],
                  dict(theta=30., phi=10.), threads=1)
    _, qv, pars = workloads.core_shell_sphere_magnetic(n=3, radius_n=3, thickness_n=3)
    assert abs(qv[0][4]) + abs(qv[1][4]) == 0.0  # grid centre is q = 0
    assert_parity("core_shell_sphere", qv, pars, threads=1)
    # empty mesh range: sums are zero
    import torch
    model = load_model("sphere")
    kernel = model.make_kernel([np.array([0.1, 0.2])])
    details, values, _ = marshal(model.info, dict(radius_pd=0.1, radius_pd_n=5),
                                 [np.array([0.1, 0.2])])
    dev_d, dev_v = kernel.upload(details, values)
    with torch.cuda.stream(kernel.stream):
        res = kernel.launch("Iq", dev_d, dev_v, 0, 0, 0.0, 0)
    kernel.stream.synchronize()
    assert not res.cpu().numpy().any()


def test_small_workspace_chunks(cuda):
    """A workspace smaller than the mesh is processed in chunks with the same
    answer."""
    import torch
    name, qv, pars = workloads.cylinder_2d(n=8, radius_n=9, length_n=9,
                                           theta_n=5, phi_n=5)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    n = details.num_eval
    full_ws = model.lib.workspace_bytes("Iqxy", kernel.q_input.nq, n, 0)
    small = torch.empty(full_ws//5, dtype=torch.uint8, device=kernel.device)
    out = torch.zeros(kernel.q_input.nq + 4, dtype=torch.float64, device=kernel.device)
    with torch.cuda.stream(kernel.stream):
        ref = kernel.launch("Iqxy", dev_d, dev_v, 0, n, 0.0, 0).clone()
        model.lib.call("Iqxy", kernel.q_input.nq, 0, n, dev_d.data_ptr(),
                       dev_v.data_ptr(), kernel.q_input.q_dev.data_ptr(),
                       out.data_ptr(), 0.0, 0, small.data_ptr(), small.numel(), 0,
                       kernel.stream.cuda_stream)
    kernel.stream.synchronize()
    worst, _ = compare_raw(out.cpu().numpy(), ref.cpu().numpy()[:kernel.q_input.nq+4],
                           1, kernel.q_input.nq, 1e-13)
    assert worst <= 1.0


def test_iq_device_matches_host(cuda):
    name, qv, pars = workloads.sphere_1d(nq=200)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    host = direct_model.call_kernel(kernel, pars)
    details, values, magnetic = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    dev = kernel.Iq_device(dev_d, dev_v, details.num_eval, values[0], values[1])
    kernel.stream.synchronize()
    np.testing.assert_allclose(dev.cpu().numpy(), host, rtol=1e-14)


@pytest.mark.parametrize("name, pars, reff_mode", [
    ("sphere", dict(radius=60, radius_pd=0.1, radius_pd_n=35), 1),
    ("core_shell_sphere", dict(radius=40, radius_pd=0.2, radius_pd_n=21, thickness=10,
                               thickness_pd=0.1, thickness_pd_n=11), 2),
    ("cylinder", dict(radius=20, radius_pd=0.1, radius_pd_n=15, length=300, length_pd=0.2,
                      length_pd_n=17), 3),
])
def test_norms_in_dll_order(cuda, name, pars, reff_mode):
    """With an effective radius requested, the four norm sums (and so R_eff
    and the volume ratio P@S hands to S) equal the DLL's bit for bit, also
    when a small workspace splits the mesh into restarted chunks."""
    import torch
    q = np.logspace(-3, np.log10(0.4), 50)
    info = load_info(name)
    ref = reference_raw(name, info, [q], pars, reff_mode=reff_mode)
    ours, nout, nq, values = gpu_raw(name, [q], pars, reff_mode=reff_mode)
    np.testing.assert_array_equal(ours[nout*nq:nout*nq + 4], ref[nout*nq:nout*nq + 4])
    model = load_model(name)
    kernel = model.make_kernel([q])
    details, values, _ = marshal(model.info, pars, [q])
    dd, dv = kernel.upload(details, values)
    n = details.num_eval
    small = model.lib.workspace_bytes("Iq", kernel.q_input.nq, 300, 0)
    ws = torch.empty(small, dtype=torch.uint8, device=kernel.device)
    out = torch.zeros(nout*nq + 4, dtype=torch.float64, device=kernel.device)
    with torch.cuda.stream(kernel.stream):
        model.lib.call("Iq", kernel.q_input.nq, 0, n, dd.data_ptr(), dv.data_ptr(),
                       kernel.q_input.q_dev.data_ptr(), out.data_ptr(), 0.0, reff_mode,
                       ws.data_ptr(), ws.numel(), 0, kernel.stream.cuda_stream)
    kernel.stream.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy()[nout*nq:], ref[nout*nq:nout*nq + 4])


def test_more_edge_cases(cuda):
    """No q points at all; a cutoff above every weight (all points dropped:
    zero norms, I = background as in the DLL); a restart that continues an
    empty first range."""
    from sasmodels_b200.direct_model import call_kernel
    model = load_model("sphere")
    kernel = model.make_kernel([np.zeros(0)])
    assert kernel.q_input.nq == 0
    assert len(call_kernel(kernel, dict(radius=50, radius_pd=0.1, radius_pd_n=5))) == 0
    q = np.array([0.01, 0.1])
    pars = dict(radius=50, radius_pd=0.1, radius_pd_n=5, background=0.25)
    assert_parity("sphere", [q], pars, cutoff=1.0, threads=1)
    kernel = model.make_kernel([q])
    np.testing.assert_array_equal(call_kernel(kernel, pars, cutoff=1.0), [0.25, 0.25])


def test_hoisted_cylinder_matches_plugin_form(cuda):
    """The cylinder library's Iqxy (per-point work hoisted out of the q loop,
    fewer divisions in J1) against the plugin's C as translated
    (sasb200_cylinder_plugin_Iqxy), over the whole +/-0.3 1/A grid with a
    reduced mesh, and both against the DLL on a strided sample."""
    import torch
    from sasmodels_b200 import _abi
    name, qv, pars = workloads.cylinder_2d(n=64, radius_n=7, length_n=5, theta_n=5,
                                           phi_n=4)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    dev_d, dev_v = kernel.upload(details, values)
    plugin = _abi.load_library(name, form="plugin")
    nq, n = kernel.q_input.nq, details.num_eval
    out = torch.zeros(nq + 4, dtype=torch.float64, device=kernel.device)
    with torch.cuda.stream(kernel.stream):
        fast = kernel.launch("Iqxy", dev_d, dev_v, 0, n, 0.0, 0).clone()
        ws = torch.empty(plugin.workspace_bytes("Iqxy", nq, n, 0), dtype=torch.uint8,
                         device=kernel.device)
        plugin.call("Iqxy", nq, 0, n, dev_d.data_ptr(), dev_v.data_ptr(),
                    kernel.q_input.q_dev.data_ptr(), out.data_ptr(), 0.0, 0,
                    ws.data_ptr(), ws.numel(), 0, kernel.stream.cuda_stream)
    kernel.stream.synchronize()
    worst, f2rel = compare_raw(fast.cpu().numpy()[:nq + 4], out.cpu().numpy(), 1, nq, 1e-12)
    assert worst <= 1.0, (worst, f2rel)
    assert_parity(name, qv, pars)


def test_fused_magnetic_matches_plugin_form(cuda):
    """core_shell_sphere Imagnetic with the spin channels sharing one
    evaluation of the Bessel terms against the plugin's C called per
    channel (sasb200_core_shell_sphere_plugin_Imagnetic), on the magnetic
    headline's grid at a reduced mesh; and against the DLL."""
    import torch
    from sasmodels_b200 import _abi
    name, qv, pars = workloads.core_shell_sphere_magnetic(n=48, radius_n=9, thickness_n=5)
    model = load_model(name)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    assert magnetic
    dev_d, dev_v = kernel.upload(details, values)
    plugin = _abi.load_library(name, form="plugin")
    nq, n = kernel.q_input.nq, details.num_eval
    out = torch.zeros(nq + 4, dtype=torch.float64, device=kernel.device)
    with torch.cuda.stream(kernel.stream):
        fused = kernel.launch("Imagnetic", dev_d, dev_v, 0, n, 0.0, 0).clone()
        ws = torch.empty(max(plugin.workspace_bytes("Imagnetic", nq, n, 0), 256),
                         dtype=torch.uint8, device=kernel.device)
        plugin.call("Imagnetic", nq, 0, n, dev_d.data_ptr(), dev_v.data_ptr(),
                    kernel.q_input.q_dev.data_ptr(), out.data_ptr(), 0.0, 0,
                    ws.data_ptr(), ws.numel(), 0, kernel.stream.cuda_stream)
    kernel.stream.synchronize()
    worst, f2rel = compare_raw(fused.cpu().numpy()[:nq + 4], out.cpu().numpy(), 1, nq, 1e-12)
    assert worst <= 1.0, (worst, f2rel)
    assert_parity(name, qv, pars)
