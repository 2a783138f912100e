"""
Generate the golden fixtures in this directory from the reference package.

    PYTHONPATH=<sasmodels source tree> python tests/golden/make_golden.py

Writes, per model, ``<model>.json`` holding

* ``tests``: the model's own embedded test cases (``models/<model>.py``
  ``tests`` lists: parameters, q or (qx, qy) points, expected I or the
  (F, F^2, R_eff, V, V_ratio) 7-tuple), excluding product (@S) cases;
* ``marshal``: for a few parameter sets, the int32 details buffer, the packed
  values vector and the magnetic flag produced by the reference's
  ``direct_model.get_mesh`` + ``details.make_kernel_args``;
* ``dll``: raw result vectors of the reference DLL (``kerneldll.DllKernel``)
  on seeded inputs, used to pin ``oracle/`` without the reference present;

and ``models_all.json``: for every C model plugin, its embedded test cases
with the reference DLL's raw result vector on each.

Run where the reference source tree is importable; the tests read only the
JSON output.
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
os.environ.setdefault("SAS_OPENCL", "none")

MODELS = ["sphere", "cylinder", "core_shell_sphere", "ellipsoid",
          "core_shell_cylinder"]


def _q_of(x):
    if not isinstance(x, list):
        x = [x]
    if isinstance(x[0], tuple):
        qx, qy = zip(*x)
        return "2d", [list(map(float, qx)), list(map(float, qy))]
    return "1d", [list(map(float, x))]


def _num(v):
    if v is None:
        return None
    if isinstance(v, (list, tuple)):
        return [_num(u) for u in v]
    return float(v)


def model_tests(info):
    out = []
    for t in info.tests or []:
        pars = t[0]
        if any(k.startswith("@") for k in pars):
            continue
        if len(t) not in (3, 7):
            continue
        kind, q = _q_of(t[1])
        case = dict(pars=pars, dim=kind, q=q)
        y = t[2] if isinstance(t[2], list) else [t[2]]
        if len(t) == 3:
            case.update(kind="I", y=_num(y))
        else:
            y2 = t[3] if isinstance(t[3], list) else [t[3]]
            case.update(kind="Fq", F=_num(y), F2=_num(y2), reff=_num(t[4]),
                        volume=_num(t[5]), volume_ratio=_num(t[6]))
        out.append(case)
    return out


def marshal_cases(name):
    from sasmodels_b200 import workloads
    cases = []
    if name == "sphere":
        _, qv, pars = workloads.sphere_1d(nq=17)
        cases.append(("1d", qv, pars))
        cases.append(("1d", qv, dict(radius=120., radius_pd=0.2, radius_pd_n=45,
                                     radius_pd_type="schulz")))
    elif name == "cylinder":
        _, qv, pars = workloads.cylinder_2d(n=6)
        cases.append(("2d", qv, pars))
        cases.append(("1d", [np.logspace(-3, -0.3, 19)],
                      dict(radius=30., radius_pd=0.15, radius_pd_n=11,
                           length=300., length_pd=0.1, length_pd_n=9,
                           length_pd_type="lognormal")))
    elif name == "core_shell_sphere":
        _, qv, pars = workloads.core_shell_sphere_magnetic(n=5, radius_n=7,
                                                           thickness_n=5)
        cases.append(("2d", qv, pars))
        cases.append(("1d", [np.logspace(-3, -0.5, 23)],
                      dict(radius=40., radius_pd=0.1, radius_pd_n=9,
                           thickness=7., thickness_pd=0.2, thickness_pd_n=5,
                           thickness_pd_type="rectangle")))
    elif name == "ellipsoid":
        cases.append(("1d", [np.logspace(-3, np.log10(0.6), 29)],
                      dict(radius_polar=30., radius_polar_pd=0.1,
                           radius_polar_pd_n=7, radius_equatorial=250.,
                           radius_equatorial_pd=0.2, radius_equatorial_pd_n=5)))
        x = np.linspace(-0.2, 0.2, 5)
        qx, qy = [a.ravel() for a in np.meshgrid(x, x)]
        cases.append(("2d", [qx, qy], dict(theta=30., phi=20.,
                                          theta_pd=5., theta_pd_n=5,
                                          radius_polar_pd=0.1, radius_polar_pd_n=5)))
    elif name == "core_shell_cylinder":
        cases.append(("1d", [np.logspace(-3, np.log10(0.6), 31)],
                      dict(radius=40., radius_pd=0.1, radius_pd_n=5,
                           thickness=15., length=900., length_pd=0.1,
                           length_pd_n=7)))
        x = np.linspace(-0.2, 0.2, 5)
        qx, qy = [a.ravel() for a in np.meshgrid(x, x)]
        cases.append(("2d", [qx, qy], dict(theta=45., phi=30., phi_pd=10.,
                                          phi_pd_n=5, radius_pd=0.1, radius_pd_n=5)))
    return cases


def c_models():
    """Every model plugin with C sources that loads here."""
    from sasmodels import core
    models_dir = os.path.join(os.path.dirname(core.__file__), "models")
    out = []
    for f in sorted(os.listdir(models_dir)):
        if not f.endswith(".py") or f.startswith("_"):
            continue
        name = f[:-3]
        try:
            info = core.load_model_info(name)
        except Exception:
            continue
        if info.source or getattr(info, "c_code", None):
            out.append(name)
    return out


def all_models_record():
    """Embedded tests of every C model, with the reference DLL's raw result
    for each case (tests/golden/models_all.json)."""
    from sasmodels import core, direct_model
    from sasmodels.details import make_kernel_args
    from sasmodels.product import RADIUS_MODE_ID
    record = {}
    for name in c_models():
        info = core.load_model_info(name)
        model = core.build_model(info, dtype="double", platform="dll")
        cases = []
        for case in model_tests(info):
            qv = [np.asarray(v, 'd') for v in case["q"]]
            pars = dict(case["pars"])
            pars.pop(RADIUS_MODE_ID, None)
            try:
                kernel = model.make_kernel(qv)
                mesh = direct_model.get_mesh(info, pars, dim=kernel.dim)
                details, values, magnetic = make_kernel_args(kernel, mesh)
                kernel._call_kernel(details, values, 0., magnetic, 0)
            except Exception:
                continue
            nout = 2 if info.have_Fq and case["dim"] == "1d" else 1
            nq = len(qv[0])
            case["raw"] = kernel.result[:nout*nq].tolist() + \
                kernel.result[nout*nq:nout*nq + 4].tolist()
            case["magnetic"] = bool(magnetic)
            cases.append(case)
        record[name] = cases
        print(name, len(cases), "cases")
    with open(os.path.join(HERE, "models_all.json"), "w") as fid:
        json.dump(record, fid, indent=0)


def main():
    from sasmodels import core, direct_model
    from sasmodels.details import make_kernel_args
    all_models_record()
    for name in MODELS:
        info = core.load_model_info(name)
        model = core.build_model(info, dtype="double", platform="dll")
        record = dict(model=name, tests=model_tests(info), marshal=[], dll=[])
        for dim, qv, pars in marshal_cases(name):
            kernel = model.make_kernel([np.asarray(v, 'd') for v in qv])
            mesh = direct_model.get_mesh(info, pars, dim=kernel.dim)
            details, values, magnetic = make_kernel_args(kernel, mesh)
            kernel._call_kernel(details, values, 0., magnetic, 0)
            nout = 2 if info.have_Fq and dim == "1d" else 1
            nq = len(qv[0])
            raw = kernel.result[:nout*nq].tolist() + \
                kernel.result[nout*nq:nout*nq + 4].tolist()
            Iq = kernel(details, values, 0., magnetic).tolist()
            entry = dict(dim=dim, q=[list(map(float, v)) for v in qv],
                         pars={k: (v if isinstance(v, str) else float(v))
                               for k, v in pars.items()},
                         details=details.buffer.tolist(),
                         values=values.tolist(), magnetic=bool(magnetic))
            record["marshal"].append(entry)
            record["dll"].append(dict(entry, raw=raw, Iq=Iq))
        with open(os.path.join(HERE, "%s.json" % name), "w") as fid:
            json.dump(record, fid, indent=0)
        print(name, len(record["tests"]), "tests,", len(record["dll"]), "dll cases")


if __name__ == "__main__":
    main()
