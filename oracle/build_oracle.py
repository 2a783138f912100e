"""
Build recipe for the CPU restatement oracle (test infrastructure only).

For each model, writes a C translation unit made of

* oracle/sas_host.h (the C99 platform layer),
* the model plugin's own C sources, read from the sasmodels package,
* a small binding (ORACLE_* macros, oracle_* functions) that maps the
  model's functions onto a flat parameter vector,
* oracle/sas_oracle.c (the restated driver),

and compiles it with the reference DLL's flags plus OpenMP into
``oracle/_build/liboracle_<model>.so`` (exported: ``oracle_kernel``).

The same model sources and binding are also compiled as C++ around
oracle/sasflops.hpp (the SAS-flop counting arithmetic) and
oracle/sasflops_driver.hpp into ``oracle/_build/libsasflops_<model>.so``
(exported: ``sasflops_count``), the instrumented restatement that sizes the
roofline numerator (driven by oracle/sasflops.py).  The generated sources
stay in the git-ignored build folder.

    python oracle/build_oracle.py [model ...] [--sasmodels PATH]
"""

import argparse
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
DEFAULT_MODELS = ["sphere", "cylinder", "core_shell_sphere", "ellipsoid",
                  "core_shell_cylinder"]


def _default_sasmodels():
    """$SASMODELS_PATH, a sasmodels checkout beside this repository, or an
    importable package (sasmodels_b200.build.locate_sasmodels)."""
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    from sasmodels_b200.build import locate_sasmodels
    return locate_sasmodels()


DEFAULT_SASMODELS = None
_IDENT = re.compile(r"(?<![.0-9A-Za-z_])([A-Za-z_][A-Za-z0-9_]*)")
_IQXY = re.compile(r"(^|\s)double\s+I(q(ac|abc|xy))\s*[(]", re.M)
_SHELL = re.compile(r"(^|\s)double\s+shell_volume\s*[(]", re.M)


def _slots(table):
    out, off = {}, 0
    for p in table.kernel_parameters:
        out[p.id] = (off, p.length)
        off += p.length
    return out


def _refs(pars, slots):
    return ", ".join(("v[%d]" % slots[p.id][0]) if slots[p.id][1] == 1
                     else "(v+%d)" % slots[p.id][0] for p in pars)


def _strfn(name, decl, body):
    return "static double %s(%s) {\n    %s\n}\n" % (name, decl or "void", body)


def _decl(pars):
    return ", ".join(("const double *%s" % p.id) if p.length > 1 else
                     "double %s" % p.id for p in pars)


def binding(info, codes):
    t = info.parameters
    slots = _slots(t)
    extra = []
    if isinstance(info.form_volume, str):
        extra.append(_strfn("form_volume", _decl(t.form_volume_parameters), info.form_volume))
    if isinstance(info.shell_volume, str):
        extra.append(_strfn("shell_volume", _decl(t.form_volume_parameters), info.shell_volume))
    if isinstance(info.Iq, str):
        extra.append(_strfn("Iq", ", ".join(["double q"] + ([_decl(t.iq_parameters)] if t.iq_parameters else [])), info.Iq))
    if isinstance(info.Iqac, str):
        extra.append(_strfn("Iqac", ", ".join(["double qab", "double qc"] + ([_decl(t.iq_parameters)] if t.iq_parameters else [])), info.Iqac))
    if isinstance(info.Iqabc, str):
        extra.append(_strfn("Iqabc", ", ".join(["double qa", "double qb", "double qc"] + ([_decl(t.iq_parameters)] if t.iq_parameters else [])), info.Iqabc))
    if isinstance(info.Iqxy, str):
        extra.append(_strfn("Iqxy", ", ".join(["double qx", "double qy"] + ([_decl(t.iq_parameters + t.orientation_parameters)])), info.Iqxy))
    alltext = codes + extra
    mode = "qa"
    for c in alltext:
        m = _IQXY.search(c)
        if m:
            mode = m.group(2)
            break
    xy = {"qa": 1, "qac": 2, "qabc": 3, "qxy": 4}[mode]
    shell = any(_SHELL.search(c) for c in alltext)
    iq = _refs(t.iq_parameters, slots)
    sep = ", " if iq else ""
    vol = _refs(t.form_volume_parameters, slots)
    mags = [k - 2 for k, p in enumerate(t.call_parameters) if p.type == "sld"]
    L = ["#define ORACLE_NPARS %d" % t.npars,
         "#define ORACLE_MAX_PD %d" % t.max_pd,
         "#define ORACLE_NVALUES %d" % t.nvalues,
         "#define ORACLE_NMAG %d" % t.nmagnetic,
         "#define ORACLE_XY %d" % xy,
         "#define ORACLE_HAVE_FQ %d" % int(bool(info.have_Fq)),
         "#define ORACLE_THETA_PAR %d" % t.theta_offset,
         "#define ORACLE_HAVE_THETA %d" % int(bool(t.orientation_parameters)),
         "#define ORACLE_HAVE_PSI %d" % int(bool(t.is_asymmetric))]
    L.append("static int oracle_mag_par(int k) { static const int m[] = {%s}; return m[k]; }"
             % (", ".join(map(str, mags)) or "0"))
    if info.valid:
        expr = _IDENT.sub(lambda m: ("(v[%d])" % slots[m.group(1)][0])
                          if m.group(1) in slots else m.group(1), info.valid)
        L.append("static int oracle_valid(const double *v) { return (%s); }" % expr)
    else:
        L.append("static int oracle_valid(const double *v) { (void)v; return 1; }")
    if t.form_volume_parameters:
        if shell:
            L.append("static void oracle_volume(const double *v, double *f, double *s)"
                     " { *f = form_volume(%s); *s = shell_volume(%s); }" % (vol, vol))
        else:
            L.append("static void oracle_volume(const double *v, double *f, double *s)"
                     " { *f = *s = form_volume(%s); }" % vol)
        if info.radius_effective_modes:
            L.append("static double oracle_reff(int mode, const double *v)"
                     " { return radius_effective(mode, %s); }" % vol)
        else:
            L.append("static double oracle_reff(int mode, const double *v)"
                     " { (void)mode; (void)v; return 0.0; }")
    else:
        L.append("static void oracle_volume(const double *v, double *f, double *s)"
                 " { (void)v; *f = *s = 1.0; }")
        L.append("static double oracle_reff(int mode, const double *v)"
                 " { (void)mode; (void)v; return 0.0; }")
    if info.have_Fq:
        L.append("static void oracle_fq(double q, double *F1, double *F2, const double *v)"
                 " { Fq(q, F1, F2%s%s); }" % (sep, iq))
        L.append("static double oracle_iq(double q, const double *v)"
                 " { double F1, F2; Fq(q, &F1, &F2%s%s); return F2; }" % (sep, iq))
    else:
        L.append("static void oracle_fq(double q, double *F1, double *F2, const double *v)"
                 " { *F1 = 0.0; *F2 = Iq(q%s%s); }" % (sep, iq))
        L.append("static double oracle_iq(double q, const double *v)"
                 " { return Iq(q%s%s); }" % (sep, iq))
    L.append("static double oracle_iqac(double a, double c, const double *v) { %s }"
             % (("return Iqac(a, c%s%s);" % (sep, iq)) if mode == "qac"
                else "(void)a; (void)c; (void)v; return 0.0;"))
    L.append("static double oracle_iqabc(double a, double b, double c, const double *v) { %s }"
             % (("return Iqabc(a, b, c%s%s);" % (sep, iq)) if mode == "qabc"
                else "(void)a; (void)b; (void)c; (void)v; return 0.0;"))
    if mode == "qxy":
        refs = ", ".join(r for r in (iq, _refs(t.orientation_parameters, slots)) if r)
        L.append("static double oracle_iqxy(double x, double y, const double *v)"
                 " { return Iqxy(x, y%s%s); }" % (", " if refs else "", refs))
    else:
        L.append("static double oracle_iqxy(double x, double y, const double *v)"
                 " { (void)x; (void)y; (void)v; return 0.0; }")
    return "\n".join(extra + L) + "\n", dict(xy=mode, have_shell=shell)


def build(models, sasmodels_path=DEFAULT_SASMODELS):
    sasmodels_path = sasmodels_path or _default_sasmodels()
    if sasmodels_path is None:
        raise RuntimeError("sasmodels sources not found: set SASMODELS_PATH")
    if sasmodels_path not in sys.path:
        sys.path.insert(0, sasmodels_path)
    os.environ.setdefault("SAS_OPENCL", "none")
    from sasmodels import core, generate
    os.makedirs(OUT, exist_ok=True)
    built = []
    for name in models:
        info = core.load_model_info(name)
        paths = generate.model_sources(info)
        codes = [open(p).read() for p in paths]
        if info.c_code:
            codes.append(info.c_code)
        bind, meta = binding(info, codes)
        unit = ["#define FLOAT_SIZE 8", '#include "sas_host.h"'] + codes + \
            [bind, '#include "sas_oracle.c"']
        c_path = os.path.join(OUT, "oracle_%s.c" % name)
        with open(c_path, "w") as fid:
            fid.write("\n".join(unit))
        so = os.path.join(OUT, "liboracle_%s.so" % name)
        cmd = ["/usr/bin/gcc", "-std=c99", "-O2", "-Wall", "-Wno-unused-function",
               "-fopenmp", "-fPIC", "-shared", "-I", HERE, c_path, "-o", so, "-lm"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode:
            raise RuntimeError("oracle compile failed for %s:\n%s" % (name, proc.stderr))
        with open(os.path.join(OUT, "oracle_%s.json" % name), "w") as fid:
            json.dump(meta, fid)
        built.append(so)
        built.append(_build_counter(name, codes, bind))
    return built


def _build_counter(name, codes, bind):
    """The SAS-flop counting library of one model (C++, OpenMP)."""
    unit = ["#define FLOAT_SIZE 8", '#include "sasflops.hpp"'] + codes + \
        [bind, '#include "sasflops_driver.hpp"']
    cpp = os.path.join(OUT, "sasflops_%s.cpp" % name)
    with open(cpp, "w") as fid:
        fid.write("\n".join(unit))
    so = os.path.join(OUT, "libsasflops_%s.so" % name)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared",
           "-Wno-unused-function", "-I", HERE, cpp, "-o", so, "-lm"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode:
        raise RuntimeError("SAS-flop counter compile failed for %s:\n%s"
                           % (name, proc.stderr[-6000:]))
    return so


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("models", nargs="*")
    ap.add_argument("--sasmodels", default=DEFAULT_SASMODELS)
    args = ap.parse_args(argv)
    for so in build(args.models or DEFAULT_MODELS, args.sasmodels):
        print(so)


if __name__ == "__main__":
    main()
