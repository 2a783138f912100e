"""
Generate ``product.json`` from the reference package: for several P@S
products, the reference's combined parameter names, its marshaled details
and values vectors (direct_model.get_mesh + details.make_kernel_args) and
the I(q) of its own ProductKernel over the reference DLLs
(direct_model.call_kernel), on seeded parameters.

    PYTHONPATH=<sasmodels source tree> python tests/golden/make_product_golden.py
"""

import json
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
os.environ.setdefault("SAS_OPENCL", "none")
os.environ.setdefault("SAS_DLL_PATH", tempfile.mkdtemp())
os.environ.setdefault("CC", "/usr/bin/gcc")

CASES = [
    ("sphere@hardsphere", "1d", dict(radius=60, radius_pd=0.1, radius_pd_n=15,
                                     volfraction=0.3, radius_effective_mode=1)),
    ("sphere@hardsphere", "1d", dict(radius=60, radius_pd=0.1, radius_pd_n=15,
                                     volfraction=0.3, structure_factor_mode=1,
                                     radius_effective_mode=1)),
    ("core_shell_sphere@hardsphere", "1d", dict(radius=40, thickness=10, thickness_pd=0.2,
                                                thickness_pd_n=11, volfraction=0.2,
                                                structure_factor_mode=1,
                                                radius_effective_mode=2)),
    ("cylinder@hayter_msa", "1d", dict(radius=20, length=120, length_pd=0.1, length_pd_n=9,
                                       volfraction=0.05, radius_effective_mode=0,
                                       radius_effective=30, charge=15)),
    ("ellipsoid@squarewell", "1d", dict(radius_polar=30, radius_equatorial=60,
                                        volfraction=0.1, radius_effective_mode=1,
                                        structure_factor_mode=1)),
    ("cylinder@hardsphere", "2d", dict(radius=20, length=100, theta=30, phi=20,
                                       radius_pd=0.1, radius_pd_n=7, volfraction=0.15,
                                       radius_effective_mode=1)),
]


def main():
    from sasmodels import core, details, direct_model
    out = []
    for name, dim, pars in CASES:
        info = core.load_model_info(name)
        model = core.build_model(info, dtype="double", platform="dll")
        if dim == "1d":
            qv = [np.logspace(-3, np.log10(0.5), 120)]
        else:
            x = np.linspace(-0.2, 0.2, 11)
            qv = [a.ravel() for a in np.meshgrid(x, x + 0.003)]
        kernel = model.make_kernel(qv)
        I = direct_model.call_kernel(kernel, dict(pars))
        mesh = direct_model.get_mesh(info, dict(pars), dim=dim)
        call_details, values, magnetic = details.make_kernel_args(kernel, mesh)
        out.append(dict(name=name, dim=dim, pars=pars, q=[v.tolist() for v in qv],
                        call_parameters=[p.name for p in info.parameters.call_parameters],
                        details=call_details.buffer.astype(int).tolist(),
                        values=values.tolist(), I=np.asarray(I).tolist()))
        kernel.release()
    with open(os.path.join(HERE, "product.json"), "w") as fid:
        json.dump(out, fid)


if __name__ == "__main__":
    main()
