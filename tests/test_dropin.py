"""
The drop-in boundary the way the reference's own callers use it.

``sasmodels_b200.install()`` wraps ``sasmodels.core.build_model``; after it
the reference's ``core.load_model``/``build_model`` (``core.py:117-128,
293-341``), ``direct_model.call_kernel``/``call_Fq`` (``direct_model.py:41-77``)
and ``DirectModel.__call__`` (``direct_model.py:354-373``) run unchanged on
the B200 engine.  These tests drive those reference functions and compare
with the reference's own DLL platform through the same functions.

They need the sasmodels package importable (``$SASMODELS_PATH``, a checkout
beside this repository, or an installed sasmodels) and are skipped where it
is absent.  On CPU the engine's device launch is replaced by the reference
DLL (``OracleKernel``), so what is checked there is the glue: routing,
the reference's marshaling of our kernel's attributes, our normalisation and
result layout; the results must then equal the reference's bit for bit.  The
``gpu`` test runs the real sm_100a kernels at the 1e-12 bar.
"""

import os
import sys

import numpy as np
import pytest

from helpers import RTOL_FP64, interleave, nout_of
from sasmodels_b200 import core as b200core
from sasmodels_b200.build import locate_sasmodels
from sasmodels_b200.kernel import B200Kernel, B200Model

SASMODELS = locate_sasmodels()
needs_sasmodels = pytest.mark.skipif(
    SASMODELS is None, reason="sasmodels package not importable (set SASMODELS_PATH)")


@pytest.fixture
def reference(monkeypatch, tmp_path):
    """The reference package with install() applied; its DLL platform builds
    into a temporary directory."""
    if SASMODELS not in sys.path:
        monkeypatch.syspath_prepend(SASMODELS)
    monkeypatch.setenv("SAS_DLL_PATH", str(tmp_path / "dll"))
    monkeypatch.setenv("SAS_OPENCL", "none")
    if os.path.exists("/usr/bin/gcc"):
        monkeypatch.setenv("CC", "/usr/bin/gcc")
    import sasmodels.core
    import sasmodels.direct_model
    b200core.install()
    yield sasmodels
    b200core.uninstall()


def _cases():
    x = np.linspace(-0.3, 0.3, 7)
    qx, qy = [a.ravel() for a in np.meshgrid(x, x)]
    xm = np.linspace(-0.1, 0.1, 5)
    mx, my = [a.ravel() for a in np.meshgrid(xm, xm)]
    return [
        ("sphere", [np.logspace(-3, np.log10(0.5), 40)],
         dict(radius=50., radius_pd=0.1, radius_pd_n=35, sld=4., sld_solvent=1.,
              background=0.001)),
        ("cylinder", [qx, qy],
         dict(radius=20., radius_pd=0.1, radius_pd_n=7, length=400., length_pd=0.1,
              length_pd_n=5, theta=60., phi=60., theta_pd=10., theta_pd_n=5,
              phi_pd=15., phi_pd_n=4, sld=4., sld_solvent=1., background=0.001)),
        ("core_shell_sphere", [mx, my],
         dict(radius=60., radius_pd=0.2, radius_pd_n=9, radius_pd_type="lognormal",
              thickness=10., thickness_pd=0.1, thickness_pd_n=5,
              sld_core_M0=1.5, sld_core_mtheta=30., sld_core_mphi=70.,
              sld_shell_M0=0.5, sld_shell_mtheta=120., sld_shell_mphi=200.,
              up_frac_i=0.9, up_frac_f=0.8, up_theta=90., up_phi=45.)),
        ("ellipsoid", [np.logspace(-3, np.log10(0.6), 30)],
         dict(radius_polar=30., radius_polar_pd=0.1, radius_polar_pd_n=9,
              radius_equatorial=200., sld=2., sld_solvent=6.)),
    ]


class OracleKernel(B200Kernel):
    """A B200Kernel whose device launch is replaced by the reference DLL
    (oracle/_ref): everything else -- attributes, Iq/Fq normalisation,
    result layout, q handling -- is the engine's own code."""

    def __init__(self, model, q_vectors, device=None, reorder=True):
        self.model = model
        self.info = model.info
        self.meta = model.meta
        self.dtype = model.dtype
        self.q_input = _HostQ(q_vectors)
        self.dim = '2d' if len(q_vectors) == 2 else '1d'
        nout = 2 if self.meta.have_Fq else 1
        self.result = np.empty(self.q_input.nq*nout + 4, 'd')

    def _call_kernel(self, call_details, values, cutoff, magnetic, radius_effective_mode):
        from oracle import refdll
        nout = nout_of(self.meta, self.dim)
        variant = "Iq" if self.dim == '1d' else ("Imagnetic" if magnetic else "Iqxy")
        q = interleave(self.q_input.q_vectors)
        raw = refdll.load(self.meta.id).call(variant, q, call_details.buffer, values,
                                             nout, cutoff, radius_effective_mode)
        self.result[:raw.size] = raw

    def release(self):
        pass


class _HostQ:
    def __init__(self, q_vectors):
        self.q_vectors = [np.ascontiguousarray(v, 'd').ravel() for v in q_vectors]
        self.nq = int(self.q_vectors[0].size)


def _dll_model(sasmodels, name):
    return sasmodels.core.load_model(name, dtype="double", platform="dll")


@needs_sasmodels
def test_install_routes_platform_b200(reference):
    """platform="b200" and SAS_OPENCL=b200 reach this backend; the caller's
    own ModelInfo comes back as the model's info; other platforms still
    reach the reference's builders."""
    sc = reference.core
    info = sc.load_model_info("cylinder")
    model = sc.build_model(info, platform="b200")
    assert isinstance(model, B200Model)
    assert model.info is info
    assert model.meta.id == "cylinder"
    model = sc.load_model("sphere", dtype="double", platform="b200")
    assert isinstance(model, B200Model) and model.info.id == "sphere"
    os.environ["SAS_OPENCL"] = "b200"
    try:
        assert isinstance(sc.build_model(info), B200Model)
    finally:
        os.environ["SAS_OPENCL"] = "none"
    dll = sc.build_model(info, platform="dll")
    assert type(dll).__module__ == "sasmodels.kerneldll"


@needs_sasmodels
def test_mixture_and_python_models_stay_reference(reference):
    """A mixture stays the reference's MixtureModel, its parts built here;
    a pure-Python model stays the reference's Python kernel."""
    sc = reference.core
    mix = sc.build_model(sc.load_model_info("sphere+cylinder"), platform="b200")
    assert type(mix).__name__ == "MixtureModel"
    assert all(isinstance(p, B200Model) for p in mix.parts)
    py_info = None
    for name in ("line", "power_law"):
        try:
            info = sc.load_model_info(name)
        except Exception:
            continue
        if not info.compiled:
            py_info = info
            break
    if py_info is not None:
        assert not isinstance(sc.build_model(py_info, platform="b200"), B200Model)


@needs_sasmodels
@pytest.mark.parametrize("case", range(4))
def test_reference_callers_on_engine_glue(reference, monkeypatch, case):
    """The reference's call_kernel, call_Fq and DirectModel on a B200 model
    whose device launch is the reference DLL: bit-for-bit the reference's
    own DLL platform through the same functions."""
    monkeypatch.setattr(B200Model, "make_kernel",
                        lambda self, q_vectors, reorder=True: OracleKernel(self, q_vectors))
    name, qv, pars = _cases()[case]
    sc, dm = reference.core, reference.direct_model
    ours = sc.load_model(name, dtype="double", platform="b200")
    dll = _dll_model(reference, name)
    k_ours, k_dll = ours.make_kernel(qv), dll.make_kernel(qv)
    np.testing.assert_array_equal(dm.call_kernel(k_ours, dict(pars)),
                                  dm.call_kernel(k_dll, dict(pars)))
    if len(qv) == 1:
        a = dm.call_Fq(k_ours, dict(pars, radius_effective_mode=1))
        b = dm.call_Fq(k_dll, dict(pars, radius_effective_mode=1))
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
        data = reference.data.empty_data1D(qv[0])
    else:
        data = reference.data.empty_data2D(np.unique(qv[0]), np.unique(qv[1]))
        data.mask = np.zeros_like(data.qx_data, dtype=bool)
    np.testing.assert_array_equal(dm.DirectModel(data, ours)(**pars),
                                  dm.DirectModel(data, dll)(**pars))


@needs_sasmodels
def test_single_precision_names_warn(reference):
    """dtype "single"/"fast" select the FP32-compensated form and say so."""
    with pytest.warns(UserWarning, match="FP32-compensated"):
        model = reference.core.load_model("cylinder", dtype="single", platform="b200")
    assert model.form == "float32c"
    with pytest.warns(UserWarning, match="not the plain single-precision"):
        reference.core.load_model("cylinder", dtype="fast", platform="b200")


@pytest.mark.gpu
@needs_sasmodels
@pytest.mark.parametrize("case", range(4))
def test_reference_callers_on_gpu(cuda, reference, case):
    """The same reference callers on the real sm_100a kernels: within the
    FP64 bar of the reference's DLL platform."""
    name, qv, pars = _cases()[case]
    sc, dm = reference.core, reference.direct_model
    ours = sc.load_model(name, dtype="double", platform="b200")
    dll = _dll_model(reference, name)
    k_ours, k_dll = ours.make_kernel(qv), dll.make_kernel(qv)
    np.testing.assert_allclose(dm.call_kernel(k_ours, dict(pars)),
                               dm.call_kernel(k_dll, dict(pars)), rtol=RTOL_FP64, atol=0)
    if len(qv) == 1:
        data = reference.data.empty_data1D(qv[0])
    else:
        data = reference.data.empty_data2D(np.unique(qv[0]), np.unique(qv[1]))
    np.testing.assert_allclose(dm.DirectModel(data, ours)(**pars),
                               dm.DirectModel(data, dll)(**pars), rtol=RTOL_FP64, atol=0)
