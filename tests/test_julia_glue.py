"""The Julia glue (julia/GLMMHDB200.jl) against the C ABI header, on the CPU.

Julia is not in this image, so the module is not run here.  What can be checked without it is
checked: every `ccall` in the module names a symbol that include/glmmhd_b200.h declares and the
library exports, with the same number of arguments and the same type class per argument and for
the return value; and the Julia structs mirroring gmt_params / gmt_step_args / gmt_diag list the
C fields in order with matching types.
"""
import os
import re

import pytest

from glmmhdturb_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "julia", "GLMMHDB200.jl")
HDR = os.path.join(ROOT, "include", "glmmhd_b200.h")


def _strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", " ", s, flags=re.S)


def c_class(t):
    t = t.strip()
    if "*" in t or "[" in t:
        return "cstring" if re.fullmatch(r"const\s+char\s*\*", t) else "ptr"
    t = re.sub(r"\bconst\b", "", t).strip()
    return {"int": "i32", "int32_t": "i32", "uint32_t": "u32", "double": "f64", "float": "f32", "void": "void",
            "int64_t": "i64"}[t]


def header_prototypes():
    text = _strip_c_comments(open(HDR).read())
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w \t\*]*?)\b(\w+)\s*\(([^;{()]*)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        if name in ("if", "while", "return"):
            continue
        argc = []
        if args.strip() not in ("", "void"):
            for a in args.split(","):
                a = a.strip()
                arr = "[" in a
                a = re.sub(r"\[.*\]", "", a)
                a = re.sub(r"\b\w+$", "", a).strip() if not a.endswith("*") else a   # drop the parameter name
                argc.append("ptr" if arr else c_class(a))
        protos[name] = (c_class(ret), argc)
    return protos


def jl_class(t):
    t = t.strip()
    if re.match(r"(Ptr|CuPtr|Ref)\{", t):
        return "ptr"
    return {"Cint": "i32", "Int32": "i32", "UInt32": "u32", "Float64": "f64", "Cdouble": "f64", "Cfloat": "f32",
            "Float32": "f32", "Cstring": "cstring", "Cvoid": "void", "Int64": "i64"}[t]


def julia_ccalls():
    src = open(JL).read()
    out = []
    for m in re.finditer(r"ccall\(\(:(\w+),\s*LIB\),\s*(\w+),\s*\(([^()]*)\)", src, flags=re.S):
        name, ret, args = m.group(1), m.group(2), m.group(3)
        types = [a for a in (x.strip() for x in args.replace("\n", " ").split(",")) if a]
        out.append((name, jl_class(ret), [jl_class(a) for a in types]))
    return out


def test_julia_ccalls_match_the_header():
    protos = header_prototypes()
    calls = julia_ccalls()
    assert len(calls) >= 15
    for name, ret, args in calls:
        assert name in protos, f"{name} is not declared in include/glmmhd_b200.h"
        assert name in _lib.EXPORTS, f"{name} is not exported by libglmmhd_b200.so"
        cret, cargs = protos[name]
        assert ret == cret, (name, ret, cret)
        assert args == cargs, (name, args, cargs)


def test_julia_covers_the_reference_step_api():
    src = open(JL).read()
    for fn in ("step_plm!", "step_tiled!", "step_fused!", "step_multi!", "compute_dt", "diagnostics", "ou_advance!",
               "ChainRulesCore.rrule"):
        assert re.search(r"(function|^)\s*" + re.escape(fn) + r"\(", src, flags=re.M), fn
    assert "module CTMHD" in src and re.search(r"function step!\(U, bxf, byf, bzf", src)
    for sym in ("gmt_step", "gmt_compute_dt", "gmt_ct_step", "gmt_adjoint_step", "gmt_forcing_advance"):
        assert f"(:{sym}, LIB)" in src, sym


def _c_struct_fields(name):
    text = _strip_c_comments(open(HDR).read())
    body = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + ";", text, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(\w+)\s+(.*)", decl)
        for f in m.group(2).split(","):
            fields.append((f.strip(), c_class(m.group(1))))
    return fields


def _jl_struct_fields(name):
    src = open(JL).read()
    body = re.search(r"struct " + name + r"\s*\n(.*?)\nend", src, flags=re.S).group(1)
    return [(f, jl_class(t)) for f, t in re.findall(r"(\w+)::(\w+)", body)]


@pytest.mark.parametrize("c,jl", [("gmt_params", "GmtParams"), ("gmt_step_args", "GmtStepArgs"),
                                  ("gmt_diag", "GmtDiag")])
def test_julia_structs_mirror_the_c_structs(c, jl):
    assert _jl_struct_fields(jl) == _c_struct_fields(c)
