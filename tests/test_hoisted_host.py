"""
The hand-rearranged FP64 bindings (csrc/fp64_hoisted_cylinder.cuh,
csrc/fp64_hoisted_core_shell_sphere.cuh) compiled for the host against the
plugin's own C sources and compared with the plugin's functions on random
inputs: the hoisted cylinder row evaluation against Iqac after qac_apply
(cylinder.c:92-102, kernel_iq.c:230-242) on both J1 branches, and the fused
spin channels of core_shell_sphere against one Fq call per channel
(core_shell_sphere.c:19-30).  This checks the rearranged mathematics (tables,
branches, operands) on the CPU; the device arithmetic is checked against the
reference DLL by the GPU parity tests.

Needs the sasmodels plugin sources (SASMODELS_PATH, a checkout beside this
repository, or an installed sasmodels) and g++; skipped without them.
"""

import ctypes as ct
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from sasmodels_b200.build import CSRC, locate_sasmodels

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SASMODELS = locate_sasmodels()
pytestmark = pytest.mark.skipif(SASMODELS is None or shutil.which("g++") is None,
                                reason="needs the sasmodels sources and g++")

PRELUDE = """
#define FLOAT_SIZE 8
#include "sas_host.h"
#include "fp64_recip.cuh"
#define __device__
#define __forceinline__
static inline double rsqrt(double x) { return 1.0/sqrt(x); }
"""


def _build(name, header, extra, tmp_path):
    if SASMODELS not in sys.path:
        sys.path.insert(0, SASMODELS)
    os.environ.setdefault("SAS_OPENCL", "none")
    from sasmodels import core, generate
    info = core.load_model_info(name)
    codes = [open(p).read() for p in generate.model_sources(info)]
    unit = [PRELUDE] + codes + [extra[0], '#include "%s"' % header, extra[1]]
    src = tmp_path / ("host_%s.cpp" % name)
    src.write_text("\n".join(unit))
    so = tmp_path / ("libhost_%s.so" % name)
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-w", "-I", os.path.join(ROOT, "oracle"),
           "-I", CSRC, str(src), "-o", str(so)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr[-3000:]
    return ct.CDLL(str(so))


CYLINDER = ("struct SasModel {};", r"""
extern "C" double hoisted(double qx, double qy, const double *v, const double *rot) {
    double row[6];
    SasModelHoisted::hoist_row(1.0, v, rot, row);
    return SasModelHoisted::eval_row(qx, qy, qx*qx + qy*qy, row);
}
extern "C" double plugin(double qx, double qy, const double *v, const double *rot) {
    const double qc = rot[0]*qx + rot[1]*qy;
    const double qab_sq = -qc*qc + qx*qx + qy*qy;
    const double qab = qab_sq > 0.0 ? sqrt(qab_sq) : 0.0;
    return Iqac(qab, qc, v[0], v[1], v[2], v[3]);
}
extern "C" double j1x(double x) { return SasModelHoisted::j1x(x); }
extern "C" double j1x_plugin(double x) { return sas_2J1x_x(x); }
""")


def test_hoisted_cylinder_matches_plugin_iqac(tmp_path):
    lib = _build("cylinder", "fp64_hoisted_cylinder.cuh", CYLINDER, tmp_path)
    D = ct.c_double
    P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    for fn in (lib.hoisted, lib.plugin):
        fn.argtypes, fn.restype = [D, D, P, P], D
    for fn in (lib.j1x, lib.j1x_plugin):
        fn.argtypes, fn.restype = [D], D
    # 2 J1(x)/x over both branches (x = 5 is the switch) and near its zeros
    xs = np.concatenate([np.linspace(0, 5, 2001), 5 + 1e-12*np.arange(3),
                         np.geomspace(5.0001, 2000, 4000), [3.8317059702075123, 7.0155866698156]])
    got = np.array([lib.j1x(x) for x in xs])
    want = np.array([lib.j1x_plugin(x) for x in xs])
    scale = np.maximum(np.abs(want), 1e-3*np.abs(want).max()*np.exp(-xs/50))
    assert np.max(np.abs(got - want)/scale) < 1e-13
    # a term near a zero of J1 or of the sinc is tiny and carries a large
    # relative error in both forms; what enters a mesh sum of non-negative
    # terms is the error against the term's envelope 1e-4 (drho V)^2
    rng = np.random.default_rng(5)
    worst = 0.0
    big = 0
    for _ in range(4000):
        v = np.array([rng.uniform(-1, 7), rng.uniform(-1, 7), rng.uniform(5, 300),
                      rng.uniform(10, 3000), 0.0, 0.0])
        a = rng.uniform(0, 2*np.pi)
        s = rng.uniform(-1, 1)
        rot = np.array([np.sqrt(1 - s*s)*np.cos(a), np.sqrt(1 - s*s)*np.sin(a)])
        qx, qy = rng.uniform(-0.5, 0.5, 2)
        h, p = lib.hoisted(qx, qy, v, rot), lib.plugin(qx, qy, v, rot)
        qc = rot[0]*qx + rot[1]*qy
        big += np.sqrt(max(qx*qx + qy*qy - qc*qc, 0))*v[2] > 5
        envelope = 1e-4*((v[0] - v[1])*np.pi*v[2]**2*v[3])**2
        worst = max(worst, abs(h - p)/max(abs(p), 1e-4*envelope))
    assert big > 1000                   # the asymptotic J1 branch ran
    assert worst < 1e-12, worst


CORE_SHELL = ("struct SasModel { static int mag_par(int k) { return 2 + k; } };", r"""
extern "C" double fused(double q, const double *v, const double *eff15, const double *w) {
    double eff[5][3];
    for (int c = 0; c < 5; ++c) for (int k = 0; k < 3; ++k) eff[c][k] = eff15[3*c + k];
    return SasModelHoisted::mag_channels(q, v, eff, w);
}
extern "C" double per_channel(double q, const double *v, const double *eff15, const double *w) {
    double F2 = 0.0;
    for (int c = 0; c < 5; ++c) {
        if (!(w[c] > 0.0)) continue;
        double F1, f2;
        Fq(q, &F1, &f2, v[0], v[1], eff15[3*c], eff15[3*c + 1], eff15[3*c + 2]);
        F2 += w[c]*f2;
    }
    return F2;
}
""")


def test_fused_spin_channels_match_per_channel_fq(tmp_path):
    lib = _build("core_shell_sphere", "fp64_hoisted_core_shell_sphere.cuh", CORE_SHELL,
                 tmp_path)
    D = ct.c_double
    P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    for fn in (lib.fused, lib.per_channel):
        fn.argtypes, fn.restype = [D, P, P, P], D
    rng = np.random.default_rng(6)
    for _ in range(3000):
        v = np.array([rng.uniform(5, 200), rng.uniform(1, 50), 1.0, 2.0, 3.0])
        eff = rng.uniform(-5, 8, 15)
        w = rng.uniform(0, 1, 5)
        w[rng.uniform(size=5) < 0.2] = 0.0
        q = rng.uniform(1e-4, 0.3)
        a, b = lib.fused(q, v, eff, w), lib.per_channel(q, v, eff, w)
        assert a == b or abs(a - b) <= 1e-13*abs(b), (a, b)
