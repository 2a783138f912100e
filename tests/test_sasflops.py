"""
The SAS-flop counter (oracle/sasflops.py): the reference's own model C run
with a counting arithmetic type.  Its per-branch counts are pinned to counts
made by hand from the reference source, and the bench's table of
configuration totals to the counter.

Hand counts (SAS-flop v1: + - * compare 1, / sqrt 4, sin cos 16, sincos 24):

* sphere Fq (sphere.c:13-20, lib/sas_3j1x_x.c:46-57) plus the two
  accumulations: qr 1, fabs + compare 2; series branch q^2 1 + polynomial 6;
  else SINCOS 24 + 3 (sin/q - cos)/(q q) 11; contrast 1, 4/3 pi R^3 3,
  contrast V bes 2, 1e-2 F 1, 1e-4 F F 2; w F^2 and w F 4
  -> 23 (qr < 0.1) and 51.
* cylinder Iqac (cylinder.c:92-102, :7-11, lib/sas_J1.c:107-153, :240-245)
  with qac_apply (kernel_iq.c:230-242) and the accumulation: qac_apply 13
  (qc 3, qab^2 5, compare 1, sqrt 4), qab R 1, x != 0 1, 2 J1/x 5, J1 sign
  test 1, branch test 1; small branch z 1, polevl(3) 6, p1evl(8) 15, / 4,
  w x (z-Z1)(z-Z2) 5, sign 1; large branch 5/x 4, z 1, polevl(6) 12 x2, / 4,
  polevl(7) 14, p1evl(7) 13, / 4, SINCOS 24, p(s-c) + w q (s+c) 6, sign p c /
  sqrt 10; sin(x)/x of qc L/2: 2 + 1 + 16 + 4; J1 term x sinc 1; volume 3,
  contrast 2; 1e-4 (s F)^2 3; w F^2 2 -> 88 and 160.
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_BUILD = os.path.join(ROOT, "oracle", "_build")


def _sasflops():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sasflops
    return sasflops


def _bench():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_sphere_branch_counts():
    sf = _sasflops()
    q = np.array([1e-3, 0.5])          # q R = 0.05 (series) and 25
    out = sf.count("sphere", [q], dict(radius=50.), threads=1)
    assert out["branch_mix"] == {23: 1, 51: 1}


def test_cylinder_branch_counts():
    """One (q, point) pair per J1 branch: theta = phi = 90 puts the axis
    along qy, so qab = |qx| and qc = qy; R = 20 makes x = 0.2 and 8.  With
    the axis along qx instead (phi = 0) qab = 0: the x != 0 and qab^2 > 0
    guards skip J1 and the square root, 88 - 39 - 4 = 45."""
    sf = _sasflops()
    qx = np.array([0.01, 0.4])
    qy = np.array([1e-3, 1e-3])
    out = sf.count("cylinder", [qx, qy], dict(radius=20., length=400., theta=90., phi=90.),
                   threads=1)
    assert out["branch_mix"] == {88: 1, 160: 1}
    assert out["evals"] == 2
    out = sf.count("cylinder", [qx, qy*0], dict(radius=20., length=400., theta=90., phi=0.),
                   threads=1)
    assert out["branch_mix"] == {45: 2}


@pytest.mark.parametrize("config", ["sphere1d", "magnetic"])
def test_bench_table_matches_counter(config):
    sf = _sasflops()
    got = sf.config(config)
    want = _bench().SASFLOPS[config]
    assert (got["evals"], got["eval_sasflops"], got["point_sasflops"],
            got["q_sasflops"]) == (want["evals"], want["eval"], want["point"], want["q"])


def test_bench_cylinder_table_consistent_with_sample():
    """The headline's full-grid count (3.2e10 evaluations, minutes to
    recount) against a strided 16x16 sample of the same grid: same branch
    counts per evaluation, same per-evaluation mean within the sampling
    difference of the branch mix, and the evaluation count of the grid."""
    sf = _sasflops()
    sample = sf.config("cylinder2d_strided_16")
    want = _bench().SASFLOPS["cylinder2d"]
    assert set(sample["branch_mix"]) == {88, 160}
    assert want["evals"] == 65536*490000
    # evals * 88 + (asymptotic evals) * 72 = eval total, with an integer count
    big = (want["eval"] - 88*want["evals"])/72
    assert big == int(big) and 0.20 < big/want["evals"] < 0.23
    assert abs(sample["sasflops_per_eval"] - want["eval"]/want["evals"]) < 0.2
