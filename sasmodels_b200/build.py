"""
Build the per-model sm_100a shared libraries.

    python -m sasmodels_b200.build [model ...] [--sasmodels PATH] [--jobs N]

For each model the sasmodels plugin is loaded (parameter table + C sources),
translated by :mod:`sasmodels_b200.generate`, and compiled with nvcc into
``sasmodels_b200/lib/libsasb200_<model>.so`` with its metadata in
``sasmodels_b200/lib/<model>.json``.  The translation unit goes to
``sasmodels_b200/_build/`` (git-ignored).  Nothing is JIT-compiled at run
time, so the libraries can be copied to a GPU host without sasmodels.
"""

import argparse
import json
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

from . import generate

PKG = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(PKG, "lib")
BUILD = os.path.join(PKG, "_build")
CSRC = os.path.join(PKG, "csrc")

#: models whose libraries are always built (the measured configurations)
CORE_MODELS = ["sphere", "cylinder", "core_shell_sphere", "ellipsoid",
               "core_shell_cylinder"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]

#: models compiled without FMA contraction (``--fmad=false``), so that every
#: multiply and add rounds separately as in the x86-64 reference build (gcc
#: -O2 on baseline x86-64 has no FMA instruction to contract into).  These
#: are the ill-conditioned ones: lattice sums near the Bragg condition
#: (the paracrystals), the partial structure factors of a binary mixture,
#: and the iterative Hayter-Penfold MSA solve; with contraction their F^2
#: moves by 4e-10 .. 4e-9 relative, without it by <= 1.4e-11.  Every other
#: model meets 1e-12 with contraction and keeps the faster DFMA form.
STRICT_FP_MODELS = {"bcc_paracrystal", "fcc_paracrystal", "sc_paracrystal",
                    "binary_hard_sphere", "hayter_msa"}


def nvcc():
    path = shutil.which("nvcc")
    if path:
        return path
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found")


def nvcc_flags(extra=()):
    return ARCH_FLAGS + [
        "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-shared", "-I", CSRC,
        "--diag-suppress=177,550,549",
    ] + list(extra)


def locate_sasmodels(explicit=None):
    """
    Directory that holds the sasmodels plugin package (``<dir>/sasmodels``),
    or None.  In order: *explicit*; ``$SASMODELS_PATH``; a sasmodels
    checkout named ``reference`` beside this repository; the directory of an
    importable ``sasmodels``.  Only the build step and the tests that compare
    against the reference's own Python code need it; the built libraries run
    without it.
    """
    def ok(d):
        return bool(d) and os.path.isdir(os.path.join(d, "sasmodels"))
    for cand in (explicit, os.environ.get("SASMODELS_PATH"),
                 os.path.join(os.path.dirname(os.path.dirname(PKG)), "reference")):
        if ok(cand):
            return os.path.abspath(cand)
    try:
        import importlib.util
        spec = importlib.util.find_spec("sasmodels")
    except (ImportError, ValueError):
        spec = None
    if spec is not None and spec.origin:
        cand = os.path.dirname(os.path.dirname(spec.origin))
        if ok(cand):
            return cand
    return None


def import_sasmodels(path=None):
    """Import the sasmodels plugin package (from *path* if given)."""
    path = path or locate_sasmodels()
    if path and path not in sys.path:
        sys.path.insert(0, path)
    os.environ.setdefault("SAS_OPENCL", "none")
    import sasmodels.core  # noqa: F401
    return sys.modules["sasmodels"]


def model_sources(sm_info):
    from sasmodels import generate as sg
    paths = sg.model_sources(sm_info) if sm_info.source else []
    out = []
    for p in paths:
        with open(p) as fid:
            out.append((p, fid.read()))
    return out


def build_model(name, force=False, verbose=False, extra_flags=()):
    """Generate and compile one model; returns the library path."""
    from sasmodels import core
    sm_info = core.load_model_info(name)
    src, meta = generate.make_cuda_source(sm_info, model_sources(sm_info))
    strict = name in STRICT_FP_MODELS
    flags = nvcc_flags((["--fmad=false"] if strict else []) + list(extra_flags))
    meta["strict_fp"] = strict
    tag = generate.source_tag(src + " ".join(flags)
                              + _read(os.path.join(CSRC, "sas_driver.cuh"))
                              + _read(os.path.join(CSRC, "sas_abi.cuh"))
                              + _read(os.path.join(CSRC, "sas_device.cuh"))
                              + _read(os.path.join(CSRC, "fp64_recip.cuh"))
                              + _read(os.path.join(CSRC, "sas_noalloc.cuh"))
                              + "".join(_read(os.path.join(CSRC, h))
                                        for h in generate.HOISTED_MODELS.values())
                              + _read(os.path.join(CSRC, "fp32c_math.cuh"))
                              + _read(os.path.join(CSRC, "fp32c_models.cuh"))
                              + _read(os.path.join(CSRC, "sas_batch.cuh")))
    meta["build_tag"] = tag
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(LIB, "libsasb200_%s.so" % name)
    js = os.path.join(LIB, "%s.json" % name)
    if not force and os.path.exists(so) and os.path.exists(js):
        with open(js) as fid:
            if json.load(fid).get("build_tag") == tag:
                return so
    cu = os.path.join(BUILD, "%s.cu" % name)
    with open(cu, "w") as fid:
        fid.write(src)
    tmp = so + ".tmp"
    cmd = [nvcc()] + flags + [cu, "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (name, proc.stderr[-4000:]))
    os.replace(tmp, so)
    with open(js, "w") as fid:
        json.dump(meta, fid, indent=1)
    return so


def build_plain(cu_name, so_name, force=False, extra_flags=(), extra_deps=()):
    """Compile a model-independent .cu from csrc/ into lib/ (rebuilt when the
    source, its headers or the flags change)."""
    src = os.path.join(CSRC, cu_name)
    so = os.path.join(LIB, so_name)
    flags = nvcc_flags(extra_flags)
    tag = generate.source_tag(_read(src) + " ".join(flags)
                              + "".join(_read(os.path.join(CSRC, d)) for d in extra_deps))
    stamp = so + ".tag"
    if not force and os.path.exists(so) and os.path.exists(stamp) and _read(stamp) == tag:
        return so
    os.makedirs(LIB, exist_ok=True)
    proc = subprocess.run([nvcc()] + flags + [src, "-o", so + ".tmp"],
                          capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (cu_name, proc.stderr[-4000:]))
    os.replace(so + ".tmp", so)
    with open(stamp, "w") as fid:
        fid.write(tag)
    return so


def build_support(force=False):
    """Libraries that do not depend on a model plugin."""
    return [build_plain("peaks.cu", "libsasb200_peaks.so", force),
            build_plain("mlp.cu", "libsasb200_mlp.so", force,
                        extra_deps=("tc_ptx.cuh",)),
            build_plain("resolution.cu", "libsasb200_resolution.so", force),
            build_plain("pack.cu", "libsasb200_pack.so", force)]


def _read(path):
    with open(path) as fid:
        return fid.read()


def build(models=None, jobs=None, force=False, verbose=False, sasmodels_path=None):
    import_sasmodels(sasmodels_path)
    models = models or CORE_MODELS
    jobs = jobs or min(len(models), os.cpu_count() or 4)
    errors = {}
    with ThreadPoolExecutor(max_workers=jobs) as pool:
        futs = {m: pool.submit(build_model, m, force, verbose) for m in models}
        for m, f in futs.items():
            try:
                f.result()
            except Exception as exc:  # report all failures together
                errors[m] = str(exc)
    if errors:
        raise RuntimeError("build failed for: %s\n%s" % (
            ", ".join(errors), "\n".join(errors.values())))
    support = build_support(force)
    return [os.path.join(LIB, "libsasb200_%s.so" % m) for m in models] + support


def c_models():
    """Every model plugin with C sources that loads in the imported sasmodels."""
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
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("models", nargs="*")
    ap.add_argument("--all", action="store_true", help="every C model plugin")
    ap.add_argument("--sasmodels", default=None)
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    models = args.models or None
    if args.all:
        import_sasmodels(args.sasmodels)
        models = c_models()
    for so in build(models, args.jobs, args.force, args.verbose, args.sasmodels):
        print(so)


if __name__ == "__main__":
    main()
