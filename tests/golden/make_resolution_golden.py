"""
Generate ``resolution.json`` from the reference package's own resolution
classes (``sasmodels/resolution.py`` Pinhole1D and Slit1D,
``sasmodels/resolution2d.py`` Pinhole2D) on seeded inputs:

* 1D: measured q, widths, the reference's q_calc, a smooth positive theory
  at q_calc (a polydisperse-sphere-like curve computed here in numpy) and
  the reference's smeared result;
* slit: measured q, slit length and width, the reference's q_calc, a
  theory at q_calc and the reference's slit-smeared result;
* 2D: measured (qx, qy), (dqx, dqy), the reference's oversampling points
  and weights, a theory at those points and the reference's average.

    PYTHONPATH=<sasmodels source tree> python tests/golden/make_resolution_golden.py
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
os.environ.setdefault("SAS_OPENCL", "none")


def theory_1d(q):
    q = np.abs(q)
    x = 50.0*q
    with np.errstate(invalid="ignore", divide="ignore"):
        f = np.where(x > 1e-3, 3*(np.sin(x) - x*np.cos(x))/x**3, 1.0)
    return 1e4*f**2*np.exp(-(5.0*q)**2) + 1e-3


def theory_2d(qx, qy):
    return theory_1d(np.sqrt(qx**2 + 0.7*qy**2))


class _Data2D:
    def __init__(self, qx, qy, dqx, dqy):
        self.qx_data, self.qy_data = qx, qy
        self.q_data = np.sqrt(qx**2 + qy**2)
        self.dqx_data, self.dqy_data = dqx, dqy


def main():
    from sasmodels import resolution, resolution2d
    rng = np.random.default_rng(11)
    cases_1d = []
    for k, (nq, rel, lin) in enumerate([(100, 0.05, False), (250, 0.1, True), (60, 0.2, False),
                                       (40, 0.0, True)]):
        q = (np.linspace(0.005, 0.4, nq) if lin else np.logspace(-3, np.log10(0.5), nq))
        dq = rel*q + 1e-4*(k % 2)
        r = resolution.Pinhole1D(q, dq)
        th = theory_1d(r.q_calc)
        cases_1d.append(dict(q=q.tolist(), dq=dq.tolist(), q_calc=r.q_calc.tolist(),
                             theory=th.tolist(), result=r.apply(th).tolist()))
    cases_slit = []
    for k, (nq, length, width) in enumerate([(120, 0.05, 0.0), (80, 0.1, 0.002),
                                             (200, 0.02, 0.0005)]):
        q = np.logspace(-3, np.log10(0.3), nq)
        r = resolution.Slit1D(q, q_length=length, q_width=width)
        th = theory_1d(r.q_calc)
        cases_slit.append(dict(q=q.tolist(), q_length=length, q_width=width,
                               q_calc=r.q_calc.tolist(), theory=th.tolist(),
                               result=r.apply(th).tolist()))
    cases_2d = []
    for k, (n, acc, coords) in enumerate([(12, "Low", "polar"), (8, "Med", "polar"),
                                          (6, "Low", "cartesian")]):
        x = np.linspace(-0.2, 0.2, n) + 1e-3
        qx, qy = [a.ravel() for a in np.meshgrid(x, x + 2e-3)]
        dqx = 0.02*np.abs(qx) + 0.002
        dqy = 0.01*np.abs(qy) + 0.001*(k % 2)
        r = resolution2d.Pinhole2D(_Data2D(qx, qy, dqx.copy(), dqy.copy()), accuracy=acc,
                                   coords=coords)
        th = theory_2d(*r.q_calc)
        cases_2d.append(dict(qx=qx.tolist(), qy=qy.tolist(), dqx=dqx.tolist(), dqy=dqy.tolist(),
                             accuracy=acc, coords=coords,
                             qx_calc=r.q_calc[0].tolist(), qy_calc=r.q_calc[1].tolist(),
                             weights=r.q_calc_weights.tolist(), theory=th.tolist(),
                             result=r.apply(th).tolist()))
    with open(os.path.join(HERE, "resolution.json"), "w") as fid:
        json.dump(dict(pinhole1d=cases_1d, slit1d=cases_slit, pinhole2d=cases_2d), fid)


if __name__ == "__main__":
    main()
