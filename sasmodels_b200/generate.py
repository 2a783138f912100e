"""
Model plugin -> sm_100a CUDA translation unit.

A sasmodels model plugin is a parameter table plus C sources
(``model_info.source``, ``model_info.c_code`` and C function bodies given as
strings).  The reference turns these into one C file around its generic
driver (``sasmodels/generate.py:951-1141``).  This module does the B200
equivalent with its own machinery:

1. every model C source is run through :func:`device_source`, a small C
   lexer that marks each file-scope function ``__device__`` and moves each
   file-scope ``constant`` table into device global memory;
2. :func:`model_struct` emits a ``SasModel`` struct whose static members bind
   the model's functions to a flat parameter vector ``v[]`` (the role the
   CALL_* macros play in ``generate.py:1036-1121``);
3. the struct is handed to the hand-written driver templates in
   ``csrc/sas_driver.cuh``, which export the C-ABI entry points.

The generated ``.cu`` lives only in the build directory; model sources are
read from the installed sasmodels package at build time and never copied
into this repository.
"""

import hashlib
import json
import os
import re

from . import modelinfo as _mi

CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")

# xy mode codes shared with sas_driver.cuh
XY_CODES = {"qa": 1, "qac": 2, "qabc": 3, "qxy": 4}

#: models whose library also exports the allocation-free entry point
#: sasb200_<model>_<variant>_noalloc (csrc/sas_noalloc.cuh)
NOALLOC_EXPORTS = {"cylinder": ("Iqxy", "sasb200::VAR_IQXY")}

#: models with a hand-rearranged FP64 binding (header in csrc/, struct
#: SasModelHoisted): cylinder hoists per-mesh-point work out of the q loop of
#: its 2D form; core_shell_sphere evaluates the spin channels of its magnetic
#: form together.  Their library's sasb200_<model>_* entry points use it; the
#: plugin's C as translated stays exported as sasb200_<model>_plugin_* for
#: comparison.
HOISTED_MODELS = {"cylinder": "fp64_hoisted_cylinder.cuh",
                  "core_shell_sphere": "fp64_hoisted_core_shell_sphere.cuh"}

_IQXY_RE = re.compile(r"(^|\s)double\s+I(?P<mode>q(ac|abc|xy))\s*[(]", re.M)
_SHELL_RE = re.compile(r"(^|\s)double\s+shell_volume\s*[(]", re.M)
_IDENT_RE = re.compile(r"(?<![.0-9A-Za-z_])([A-Za-z_][A-Za-z0-9_]*)")


def find_xy_mode(sources):
    """'qac', 'qabc' or 'qxy' from the first oriented I(q) definition found,
    else 'qa' (same rule as ``generate.py:865-895``)."""
    for code in sources:
        m = _IQXY_RE.search(code)
        if m is not None:
            return m.group('mode')
    return 'qa'


def has_shell_volume(sources):
    """True if the C defines ``double shell_volume(`` (``generate.py:908-917``)."""
    return any(_SHELL_RE.search(code) for code in sources)


# ---------------------------------------------------------------- C lexer ---

_TOKEN_RE = re.compile(r"""
    (?P<comment>//[^\n]*|/\*.*?\*/)
  | (?P<pp>^[ \t]*\#(?:[^\n\\]|\\.|\\\n)*)
  | (?P<str>"(?:[^"\\\n]|\\.)*"|'(?:[^'\\\n]|\\.)*')
  | (?P<ident>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<num>\.?[0-9](?:[0-9A-Za-z_.]|[eEpP][+-])*)
  | (?P<ws>\s+)
  | (?P<punct>.)
""", re.S | re.M | re.X)

_NOT_FUNCTION_WORDS = {"typedef", "struct", "union", "enum"}


def _tokens(code):
    pos = 0
    for m in _TOKEN_RE.finditer(code):
        if m.start() != pos:
            raise ValueError("lexer gap at %d" % pos)
        pos = m.end()
        yield m.lastgroup, m.group(0)


def device_source(code):
    """
    Rewrite one model C source for device compilation.

    File-scope functions (prototypes and definitions) gain ``__device__``.
    File-scope ``constant`` data becomes ``__device__ const``; other
    file-scope data gains ``__device__``.  Inside functions ``constant``
    (pointers into the tables) becomes ``const``.  Comments, strings and
    preprocessor lines pass through untouched.
    """
    out = []
    stmt = []            # tokens of the current file-scope statement
    depth = 0            # brace depth
    for kind, text in _tokens(code):
        if depth == 0 and not stmt and kind in ("ws", "comment", "pp"):
            out.append(text)
            continue
        stmt.append((kind, text))
        if kind == "punct":
            if text == "{":
                depth += 1
            elif text == "}":
                depth -= 1
                if depth == 0 and _is_function(stmt):
                    out.append(_emit(stmt))
                    stmt = []
            elif text == ";" and depth == 0:
                out.append(_emit(stmt))
                stmt = []
    if stmt:
        out.append("".join(t for _, t in stmt))
    return "".join(out)


def _is_function(stmt):
    """A file-scope statement is a function if an identifier is followed by
    '(' before any '=' or '{' at brace/paren depth zero."""
    words = [t for k, t in stmt if k == "ident"]
    if words and words[0] in _NOT_FUNCTION_WORDS:
        return False
    prev_ident = False
    for kind, text in stmt:
        if kind in ("ws", "comment"):
            continue
        if kind == "punct":
            if text == "(" and prev_ident:
                return True
            if text in "={;":
                return False
        prev_ident = kind == "ident"
    return False


def _emit(stmt):
    words = [t for k, t in stmt if k == "ident"]
    if words and words[0] in _NOT_FUNCTION_WORDS:
        # type declarations may still carry a trailing table, e.g.
        # "typedef struct {..} T;" -- leave untouched
        return "".join(t for _, t in stmt)
    if _is_function(stmt):
        body = "".join("const" if (k == "ident" and t == "constant") else t
                       for k, t in stmt)
        return "__device__ " + body
    # file-scope data: small tables (polynomial coefficients, the 20- to
    # 150-point Gauss rules) go to __constant__ memory, where warp-uniform
    # reads are served by the constant cache; large tables (500- and
    # 5000-point rules) to global memory
    if "constant" in words:
        space = "__constant__ const" if _table_size(stmt) <= CONSTANT_TABLE_MAX \
            else "__device__ const"
        return "".join(space if (k == "ident" and t == "constant")
                       else t for k, t in stmt)
    return "__device__ " + "".join(t for _, t in stmt)


#: largest file-scope table (elements) placed in __constant__ memory
CONSTANT_TABLE_MAX = 256


def _table_size(stmt):
    """Declared element count of a file-scope array ([] counts as small)."""
    toks = [t for k, t in stmt if k not in ("ws", "comment")]
    if "[" not in toks:
        return 1
    i = toks.index("[")
    inner = toks[i + 1:toks.index("]", i)]
    if not inner:
        return 0
    try:
        return int(inner[0]) if len(inner) == 1 else 1 << 30
    except ValueError:
        return 1 << 30


# ------------------------------------------------------------ model struct ---

def _param_slots(table):
    """Map kernel parameter id -> (offset into v[], length)."""
    slots, offset = {}, 0
    for p in table.kernel_parameters:
        slots[p.id] = (offset, p.length)
        offset += p.length
    return slots


def _arg_refs(pars, slots, vec="v"):
    """Call arguments for *pars*: a scalar slot, or for a vector parameter a
    pointer to its first slot (plugins declare these `double p[]`; they only
    read them)."""
    refs = []
    for p in pars:
        off, n = slots[p.id]
        refs.append("%s[%d]" % (vec, off) if n == 1
                    else "const_cast<double *>(%s + %d)" % (vec, off))
    return refs


def _fn_from_string(name, pars, body, ctype="double"):
    """C function from a body string given in the model .py (the plugin
    API lets form_volume, Iq, ... be one-line C bodies;
    ``generate.py:667-697``)."""
    decl = []
    for p in pars:
        if getattr(p, "length", 1) > 1:
            decl.append("const %s *%s" % (ctype, p.id))
        else:
            decl.append("%s %s" % (ctype, p.id))
    args = ", ".join(decl) if decl else "void"
    return "%s %s(%s) {\n    %s\n}\n" % (ctype, name, args, body)


class _Q:
    """Stand-in parameter for q, qx, qy, qab, qa, qb, qc in generated
    function signatures."""
    def __init__(self, name):
        self.id = self.name = name
        self.length = 1


def model_struct(info, table, xy_mode, have_shell, name="SasModel"):
    """
    The binding struct the driver templates call.  ``v`` is the kernel
    parameter vector (``values[2:2+npars]`` with pd values substituted).
    """
    slots = _param_slots(table)
    npars = table.npars
    iq_refs = ", ".join(_arg_refs(table.iq_parameters, slots))
    vol_pars = table.form_volume_parameters
    vol_refs = ", ".join(_arg_refs(vol_pars, slots))
    sep = ", " if iq_refs else ""
    orient = table.orientation_parameters

    theta_par = table.theta_offset
    lines = []
    a = lines.append
    a("struct %s {" % name)
    a("  static constexpr int NPARS = %d;" % npars)
    a("  static constexpr int MAX_PD = %d;" % table.max_pd)
    a("  static constexpr int NVALUES = %d;" % table.nvalues)
    a("  static constexpr int NMAG = %d;" % table.nmagnetic)
    a("  static constexpr int XY_MODE = %d;" % XY_CODES[xy_mode])
    a("  static constexpr bool HAVE_FQ = %s;" % ("true" if info.have_Fq else "false"))
    a("  static constexpr int THETA_PAR = %d;" % theta_par)
    a("  static constexpr bool HAVE_THETA = %s;" % ("true" if orient else "false"))
    a("  static constexpr bool HAVE_PSI = %s;" % ("true" if table.is_asymmetric else "false"))
    mags = [k - _mi.NUM_COMMON_PARS for k, p in enumerate(table.call_parameters)
            if p.type == 'sld']
    a("  __device__ static int mag_par(int k) {")
    a("    switch (k) {")
    for k, idx in enumerate(mags):
        a("      case %d: return %d;" % (k, idx))
    a("      default: return 0;")
    a("    }")
    a("  }")
    # validity (model_info.valid, ``generate.py:848-862``)
    valid = getattr(info, "valid", None)
    if valid:
        def sub(m):
            word = m.group(1)
            if word in slots:
                off, n = slots[word]
                return "(v[%d])" % off if n == 1 else "(v+%d)" % off
            return word
        a("  __device__ static bool valid(const double *v) { return (%s); }"
          % _IDENT_RE.sub(sub, valid))
    else:
        a("  __device__ static bool valid(const double *) { return true; }")
    # volumes (``generate.py:1036-1070``)
    if vol_pars:
        if have_shell:
            a("  __device__ static void volume(const double *v, double &form, double &shell)"
              " { form = form_volume(%s); shell = shell_volume(%s); }" % (vol_refs, vol_refs))
        else:
            a("  __device__ static void volume(const double *v, double &form, double &shell)"
              " { form = shell = form_volume(%s); }" % vol_refs)
        if info.radius_effective_modes:
            a("  __device__ static double reff(int mode, const double *v)"
              " { return radius_effective(mode, %s); }" % vol_refs)
        else:
            a("  __device__ static double reff(int, const double *) { return 0.0; }")
    else:
        a("  __device__ static void volume(const double *, double &form, double &shell)"
          " { form = shell = 1.0; }")
        a("  __device__ static double reff(int, const double *) { return 0.0; }")
    # 1D kernels
    if info.have_Fq:
        a("  __device__ static void fq(double q, double &F1, double &F2, const double *v)"
          " { Fq(q, &F1, &F2%s%s); }" % (sep, iq_refs))
        a("  __device__ static double iq(double q, const double *v)"
          " { double F1, F2; Fq(q, &F1, &F2%s%s); return F2; }" % (sep, iq_refs))
    else:
        a("  __device__ static void fq(double q, double &F1, double &F2, const double *v)"
          " { F1 = 0.0; F2 = Iq(q%s%s); }" % (sep, iq_refs))
        a("  __device__ static double iq(double q, const double *v)"
          " { return Iq(q%s%s); }" % (sep, iq_refs))
    # 2D kernels
    if xy_mode == "qac":
        a("  __device__ static double iqac(double qab, double qc, const double *v)"
          " { return Iqac(qab, qc%s%s); }" % (sep, iq_refs))
    else:
        a("  __device__ static double iqac(double, double, const double *) { return 0.0; }")
    if xy_mode == "qabc":
        a("  __device__ static double iqabc(double qa, double qb, double qc, const double *v)"
          " { return Iqabc(qa, qb, qc%s%s); }" % (sep, iq_refs))
    else:
        a("  __device__ static double iqabc(double, double, double, const double *) { return 0.0; }")
    if xy_mode == "qxy":
        orient_refs = ", ".join(_arg_refs(orient, slots))
        refs = ", ".join(r for r in (iq_refs, orient_refs) if r)
        a("  __device__ static double iqxy(double qx, double qy, const double *v)"
          " { return Iqxy(qx, qy%s%s); }" % (", " if refs else "", refs))
    else:
        a("  __device__ static double iqxy(double, double, const double *) { return 0.0; }")
    a("};")
    return "\n".join(lines)


def _string_functions(info, table):
    out = []
    fv = table.form_volume_parameters
    q = [_Q("q")]
    if isinstance(getattr(info, "form_volume", None), str):
        out.append(_fn_from_string("form_volume", fv, info.form_volume))
    if isinstance(getattr(info, "shell_volume", None), str):
        out.append(_fn_from_string("shell_volume", fv, info.shell_volume))
    if isinstance(getattr(info, "Iq", None), str):
        out.append(_fn_from_string("Iq", q + table.iq_parameters, info.Iq))
    if isinstance(getattr(info, "Iqxy", None), str):
        out.append(_fn_from_string("Iqxy", [_Q("qx"), _Q("qy")] + table.iq_parameters
                                   + table.orientation_parameters, info.Iqxy))
    if isinstance(getattr(info, "Iqac", None), str):
        out.append(_fn_from_string("Iqac", [_Q("qab"), _Q("qc")] + table.iq_parameters,
                                   info.Iqac))
    if isinstance(getattr(info, "Iqabc", None), str):
        out.append(_fn_from_string("Iqabc", [_Q("qa"), _Q("qb"), _Q("qc")]
                                   + table.iq_parameters, info.Iqabc))
    return out


def make_cuda_source(sm_info, sources):
    """
    One translation unit for model *sm_info* (a sasmodels ModelInfo).

    *sources* is ``[(path, code), ...]`` for ``model_info.source``.  Returns
    (cuda_source_text, metadata_dict).
    """
    if getattr(sm_info, "translation", None):
        raise NotImplementedError("reparameterised models are not supported")
    if not getattr(sm_info, "compiled", True) and not sources:
        raise ValueError("%s is a pure python model" % sm_info.id)
    table = sm_info.parameters
    codes = [code for _, code in sources]
    if getattr(sm_info, "c_code", None):
        codes.append(sm_info.c_code)
    strfns = _string_functions(sm_info, table)
    xy_mode = find_xy_mode(codes + strfns)
    have_shell = has_shell_volume(codes + strfns)
    if xy_mode == "qabc" and not table.is_asymmetric:
        raise ValueError("asymmetric oriented models need to define Iqabc")
    if xy_mode == "qac" and table.is_asymmetric:
        raise ValueError("symmetric oriented models need to define Iqac")

    body = ["#define FLOAT_SIZE 8", '#include "sas_device.cuh"',
            "namespace sasm {"]
    for path, code in sources:
        body.append("// ---- model source: %s" % os.path.basename(path))
        body.append(device_source(code))
    if getattr(sm_info, "c_code", None):
        body.append("// ---- c_code")
        body.append(device_source(sm_info.c_code))
    for fn in strfns:
        body.append(device_source(fn))
    body.append(model_struct(sm_info, table, xy_mode, have_shell))
    hoisted = sm_info.id in HOISTED_MODELS
    if hoisted:
        body.append('#include "%s"' % HOISTED_MODELS[sm_info.id])
    body.append("}  // namespace sasm")
    f32c = f32c_block(sm_info.id, table, codes)
    if f32c:
        body.append(f32c)
    body.append('#include "sas_driver.cuh"')
    body.append('#include "sas_abi.cuh"')
    main_binding = "sasm::SasModelHoisted" if hoisted else "sasm::SasModel"
    body.append("SASB200_EXPORT_MODEL(%s, %s)" % (sm_info.id, main_binding))
    if hoisted:
        body.append("SASB200_EXPORT_MODEL(%s_plugin, sasm::SasModel)" % sm_info.id)
    if f32c:
        body.append("SASB200_EXPORT_MODEL(%s_f32c, sasm::SasModelF32c)" % sm_info.id)
        body.append('#include "sas_batch.cuh"')
        body.append("SASB200_EXPORT_BATCH(%s, sasm::SasModel, sasm::SasModelF32c)" % sm_info.id)
    if sm_info.id in NOALLOC_EXPORTS:
        variant, var = NOALLOC_EXPORTS[sm_info.id]
        body.append('#include "sas_noalloc.cuh"')
        body.append("SASB200_EXPORT_NOALLOC(%s, %s, %s, %s)"
                    % (sm_info.id, main_binding, variant, var))
    meta = _mi.from_sasmodels(sm_info, xy_mode, have_shell)
    meta["f32c"] = bool(f32c)
    meta["hoisted"] = hoisted
    return "\n".join(body) + "\n", meta


# ------------------------------------------------------ FP32c bindings ---

#: models with hand-written FP32-compensated physics (csrc/fp32c_models.cuh):
#: expected kernel parameter order and the binding of fq/iqac to it
F32C_MODELS = {
    "sphere": (["sld", "sld_solvent", "radius"], "QuadSphere", None),
    "core_shell_sphere": (["radius", "thickness", "sld_core", "sld_shell", "sld_solvent"],
                          "QuadCoreShellSphere", None),
    "cylinder": (["sld", "sld_solvent", "radius", "length", "theta", "phi"], "QuadCylinder",
                 "return f32c::cylinder_iqac(qab, qc, v[0], v[1], v[2], v[3]);"),
    "ellipsoid": (["sld", "sld_solvent", "radius_polar", "radius_equatorial", "theta", "phi"],
                  "QuadEllipsoid",
                  "return f32c::ellipsoid_iqac(qab, qc, v[0], v[1], v[2], v[3]);"),
    "core_shell_cylinder": (["sld_core", "sld_shell", "sld_solvent", "radius", "thickness",
                             "length", "theta", "phi"], "QuadCoreShellCylinder",
                            "return f32c::core_shell_cylinder_iqac(qab, qc, v);"),
}

_GAUSS_RE = re.compile(r"constant\s+double\s+Gauss(\d+)(Z|Wt)\s*\[\s*\d*\s*\]\s*=\s*\{(.*?)\}", re.S)
_RULES = (20, 76, 500, 5000)
_M_PI_4 = 0.7853981633974483     # kernel_header.c literal


def gauss_tables(codes):
    """{n: (z, w)} parsed from the plugin's quadrature sources."""
    import numpy as np
    found = {}
    for code in codes:
        for m in _GAUSS_RE.finditer(code):
            n, kind, body = int(m.group(1)), m.group(2), m.group(3)
            body = re.sub(r"//[^\n]*", "", body)
            vals = [float(t) for t in body.replace("\n", " ").split(",") if t.strip()]
            found.setdefault(n, {})[kind] = np.array(vals[:n])
    return {n: (d["Z"], d["Wt"]) for n, d in found.items() if "Z" in d and "Wt" in d}


def _c_array(name, vals):
    return "__device__ const double %s[%d] = {%s};" % (
        name, len(vals), ",".join(repr(float(v)) for v in vals))


def f32c_block(name, table, codes):
    """FP32c binding struct for a model listed in F32C_MODELS, or '' if the
    model has no FP32c physics (or its parameter table changed)."""
    import numpy as np
    if name not in F32C_MODELS:
        return ""
    expected, fq, iqac = F32C_MODELS[name]
    if [p.id for p in table.kernel_parameters] != expected:
        raise ValueError("FP32c binding for %s expects parameters %s" % (name, expected))
    out = ['#include "fp32c_models.cuh"', "namespace sasm {"]
    rules = gauss_tables(codes)
    if all(n in rules for n in _RULES):
        for n in _RULES:
            z, w = rules[n]
            theta = z*_M_PI_4 + _M_PI_4
            out.append(_c_array("F32cZ%d" % n, z))
            out.append(_c_array("F32cW%d" % n, w))
            out.append(_c_array("F32cSin%d" % n, np.sin(theta)))
            out.append(_c_array("F32cCos%d" % n, np.cos(theta)))
    out.append("}  // namespace sasm")
    out.append("namespace f32c {")
    out.append("__device__ __forceinline__ Rule rule_for(double qr) {")
    if all(n in rules for n in _RULES):
        out.append("  if (qr < 10) return Rule{20, sasm::F32cZ20, sasm::F32cW20, sasm::F32cSin20, sasm::F32cCos20};")
        out.append("  if (qr < 100) return Rule{76, sasm::F32cZ76, sasm::F32cW76, sasm::F32cSin76, sasm::F32cCos76};")
        out.append("  if (qr < 750) return Rule{500, sasm::F32cZ500, sasm::F32cW500, sasm::F32cSin500, sasm::F32cCos500};")
        out.append("  return Rule{5000, sasm::F32cZ5000, sasm::F32cW5000, sasm::F32cSin5000, sasm::F32cCos5000};")
    else:
        out.append("  return Rule{0, nullptr, nullptr, nullptr, nullptr};")
    out.append("}")
    out.append("}  // namespace f32c")
    out.append("namespace sasm {")
    out.append("struct SasModelF32c : SasModel {")
    out.append("  using Quad = f32c::%s;" % fq)
    out.append("  __device__ static void fq(double q, double &F1, double &F2, const double *v)"
               " { f32c::quad_fq<Quad>(q, v, F1, F2); }")
    out.append("  __device__ static double iq(double q, const double *v) { double F1, F2; fq(q, F1, F2, v); return F2; }")
    if iqac:
        out.append("  __device__ static double iqac(double qab, double qc, const double *v) { %s }" % iqac)
    if name == "core_shell_sphere":
        # the spin channels of the magnetic form share the Bessel terms
        out.append("  static constexpr bool MAG_FUSED = true;")
        out.append("  __device__ static double mag_channels(double q, const double *v,"
                   " const double (*eff)[3], const double *chan_w)"
                   " { return f32c::core_shell_sphere_channels(q, v, eff, chan_w,"
                   " [](int k) { return mag_par(k); }); }")
    out.append("};")
    out.append("}  // namespace sasm")
    return "\n".join(out)


def _jsonable_tests(tests):
    out = []
    for t in tests:
        try:
            json.dumps(t)
            out.append(t)
        except TypeError:
            continue
    return out


def info_from_sasmodels(sm_info):
    """Our ModelInfo for a live sasmodels ModelInfo (reads its C sources to
    find the 2D mode)."""
    from sasmodels import generate as sg
    paths = sg.model_sources(sm_info) if getattr(sm_info, "source", None) else []
    codes = []
    for p in paths:
        with open(p) as fid:
            codes.append(fid.read())
    if getattr(sm_info, "c_code", None):
        codes.append(sm_info.c_code)
    strfns = _string_functions(sm_info, sm_info.parameters)
    meta = _mi.from_sasmodels(sm_info, find_xy_mode(codes + strfns),
                              has_shell_volume(codes + strfns))
    return _mi.ModelInfo(meta)


def source_tag(text):
    return hashlib.sha256(text.encode("utf8")).hexdigest()[:16]
