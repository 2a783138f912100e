"""
Build recipe for the reference DLL oracle (test infrastructure only).

Compiles the *unmodified* reference kernels -- the C that sasmodels'
own generator emits for a model (``sasmodels/generate.py:951-1141``:
kernel_header.c + model sources + kernel_iq.c three times) -- with the same
compiler command as ``sasmodels/kerneldll.py:131-152`` on unix
(``cc -std=c99 -O2 -Wall -fPIC -shared ... -lm``, no OpenMP), into
``oracle/_ref/sas64_<model>.so``.  The generated C is written next to it only
for the compile and then deleted; nothing from the reference lands in the
repository.

    python oracle/build_ref.py [model ...] [--sasmodels PATH]

The libraries export ``<model>_Iq``, ``<model>_Iqxy`` and
``<model>_Imagnetic`` with the ``kernel_iq.c:317-328`` signature and are
driven by ``oracle/refdll.py``.  This runs where the reference sources are
present; the built ``.so`` files travel with the repository snapshot.
"""

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
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


def cc():
    # the image's $CC may lack libm/libgomp wiring; the system gcc is the
    # one the reference's unix branch ends up invoking as "cc"
    for cand in ("/usr/bin/gcc", "/usr/bin/cc"):
        if os.path.exists(cand):
            return cand
    return "cc"


def build(models, sasmodels_path=DEFAULT_SASMODELS, force=False):
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
        so = os.path.join(OUT, "sas64_%s.so" % name)
        info = core.load_model_info(name)
        source = generate.make_source(info)["dll"]
        source = generate.convert_type(source, generate.F64)
        tag = generate.tag_source(source)
        stamp = so + ".tag"
        if not force and os.path.exists(so) and os.path.exists(stamp):
            with open(stamp) as fid:
                if fid.read().strip() == tag:
                    built.append(so)
                    continue
        c_path = os.path.join(OUT, "sas64_%s.c" % name)
        with open(c_path, "w") as fid:
            fid.write(source)
        cmd = [cc(), "-std=c99", "-O2", "-Wall", "-fPIC", "-shared",
               c_path, "-o", so, "-lm"]
        try:
            subprocess.run(cmd, check=True, capture_output=True, text=True)
        except subprocess.CalledProcessError as exc:
            raise RuntimeError("compile failed: %s\n%s" % (" ".join(cmd), exc.stderr))
        finally:
            os.unlink(c_path)
        with open(stamp, "w") as fid:
            fid.write(tag)
        built.append(so)
    return built


def c_models(sasmodels_path=DEFAULT_SASMODELS):
    """Every model plugin with C sources that loads here."""
    sasmodels_path = sasmodels_path or _default_sasmodels()
    if sasmodels_path is None:
        raise RuntimeError("sasmodels sources not found: set SASMODELS_PATH")
    if sasmodels_path not in sys.path:
        sys.path.insert(0, sasmodels_path)
    os.environ.setdefault("SAS_OPENCL", "none")
    from sasmodels import core
    models_dir = os.path.join(os.path.dirname(core.__file__), "models")
    out = []
    for f in sorted(os.listdir(models_dir)):
        if not f.endswith(".py") or f.startswith("_"):
            continue
        try:
            info = core.load_model_info(f[:-3])
        except Exception:
            continue
        if info.source or getattr(info, "c_code", None):
            out.append(f[:-3])
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("models", nargs="*")
    ap.add_argument("--sasmodels", default=DEFAULT_SASMODELS)
    ap.add_argument("--all", action="store_true", help="every C model plugin")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    models = c_models(args.sasmodels) if args.all else (args.models or DEFAULT_MODELS)
    for so in build(models, args.sasmodels, args.force):
        print(so)


if __name__ == "__main__":
    main()
