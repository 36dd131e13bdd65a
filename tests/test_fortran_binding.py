"""The Fortran ISO_C_BINDING include (include/adz_b200_f90.inc) against the C
header (include/adz_b200.h).

No Fortran compiler is available to build a caller, so the include is parsed
and checked against the header's prototypes and structs:

* every Level B entry point (adzc_*) of the header has one interface whose
  bind(C, name=...) is that symbol, and nothing else is bound;
* the arity, the argument order, the result type and, per argument, how it is
  passed: a C scalar by value with the matching kind; a single-level C pointer
  either as type(C_PTR), value (a device address) or by reference to an entity
  of the pointee's type; a C pointer to pointers (the HOST arrays of DEVICE
  pointers, out-handles) by reference as type(C_PTR);
* every bind(C) derived type has the C struct's members in order, with
  matching kinds and array extents.

This is the binding the reference keeps for its interpolator in
src/gemdyn/src/base/tricublin_f90.inc:1-80.
"""
from __future__ import annotations

import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "adz_b200.h")
INC = os.path.join(ROOT, "include", "adz_b200_f90.inc")

SCALAR_KIND = {"int": "integer(C_INT)", "double": "real(C_DOUBLE)", "float": "real(C_FLOAT)",
               "long long": "integer(C_LONG_LONG)", "char": "character(kind=C_CHAR)"}
STRUCTS = ("adzc_grid", "adzc_info", "adzc_domain", "adzc_bc_tracer", "adzc_halo")


# --------------------------------------------------------------------------- C
def _c_source():
    s = open(HDR).read()
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"^\s*#.*$", " ", s, flags=re.M)


def _c_type(decl: str):
    """'const void *const *srcs' -> ('void', 2, 'srcs'); 'float ms[3]' ->
    ('float', 1, 'ms')."""
    decl = decl.strip()
    stars = decl.count("*")
    arr = re.search(r"\[(\d*)\]\s*$", decl)
    if arr:
        stars += 1
        decl = decl[:arr.start()]
    m = re.match(r"(.*?)([A-Za-z_]\w*)\s*$", decl.replace("*", " "))
    base = " ".join(w for w in m.group(1).split() if w not in ("const", "unsigned"))
    return base, stars, m.group(2)


def c_prototypes():
    out = {}
    for ret, name, args in re.findall(r"(int|long long|const char\s*\*)\s*(adzc_\w+)\s*\(([^)]*)\)\s*;",
                                      _c_source()):
        args = args.strip()
        params = [] if args in ("", "void") else [_c_type(a) for a in args.split(",")]
        out[name] = (ret.replace(" ", ""), params)
    return out


def c_structs():
    out = {}
    for body, name in re.findall(r"typedef\s+struct\s*\{([^{}]*)\}\s*(adzc_\w+)\s*;", _c_source()):
        fields = []
        for stmt in body.split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            m = re.match(r"((?:const\s+)?(?:unsigned\s+)?(?:long long|int|double|float|void|char|adzc_\w+))(.*)",
                         stmt, flags=re.S)
            base = m.group(1).replace("const", "").strip()
            for d in m.group(2).split(","):
                d = d.strip()
                dims = re.findall(r"\[(\d+)\]", d)
                stars = d.count("*")
                nm = re.findall(r"[A-Za-z_]\w*", re.sub(r"\[\d+\]", "", d))[-1]
                fields.append((nm, base if not stars else "ptr", int(dims[0]) if dims else 0))
        out[name] = fields
    return out


# --------------------------------------------------------------------- Fortran
def _f_lines():
    joined, cur = [], ""
    for raw in open(INC):
        line = raw.split("!")[0].rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if cur:
            s = s[1:].strip() if s.startswith("&") else s
            cur += " " + s
        else:
            cur = s
        if cur.endswith("&"):
            cur = cur[:-1].rstrip()
            continue
        joined.append(cur)
        cur = ""
    return joined


def _f_decl(line: str):
    """'integer(C_INT), intent(in), optional :: mono(*)' ->
    ('integer(C_INT)', {'intent(in)', 'optional'}, [('mono', '*')])."""
    lhs, rhs = line.split("::")
    parts = [p.strip() for p in re.split(r",(?![^()]*\))", lhs)]
    names = [(m.group(1), m.group(2)) for m in re.finditer(r"(\w+)\s*(?:\(([^)]*)\))?", rhs)]
    return parts[0].replace(" ", ""), set(p.replace(" ", "") for p in parts[1:]), names


def f_interfaces():
    out, cur = {}, None
    for line in _f_lines():
        m = re.match(r"(.*?)\s*function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name='(\w+)'\)", line)
        if m:
            cur = {"result": m.group(1).replace(" ", ""), "args": [a.strip() for a in m.group(3).split(",") if
                                                                   a.strip()],
                   "bind": m.group(4), "decl": {}}
            out[m.group(2)] = cur
            continue
        if cur is not None and line.startswith("end function"):
            cur = None
            continue
        if cur is not None and "::" in line and not line.startswith("import"):
            ftype, attrs, names = _f_decl(line)
            for nm, dim in names:
                cur["decl"][nm] = (ftype, attrs, dim)
    return out


def f_types():
    out, cur = {}, None
    for line in _f_lines():
        m = re.match(r"type,\s*bind\(C\)\s*::\s*(\w+)", line)
        if m:
            cur = out.setdefault(m.group(1), [])
            continue
        if line.startswith("end type"):
            cur = None
            continue
        if cur is not None and "::" in line:
            ftype, _, names = _f_decl(line)
            for nm, dim in names:
                cur.append((nm, ftype, int(dim) if dim else 0))
    return out


# ----------------------------------------------------------------------- tests
def test_every_entry_point_is_bound_once():
    c, f = c_prototypes(), f_interfaces()
    assert len(c) >= 40
    assert {v["bind"] for v in f.values()} == set(c)
    for name, v in f.items():
        assert v["bind"] == name


@pytest.mark.parametrize("name", sorted(c_prototypes()))
def test_interface_matches_prototype(name):
    ret, params = c_prototypes()[name]
    fi = f_interfaces()[name]
    want_ret = {"int": "integer(C_INT)", "longlong": "integer(C_LONG_LONG)", "constchar*": "type(C_PTR)"}[ret]
    assert fi["result"] == want_ret
    assert len(fi["args"]) == len(params), (fi["args"], params)
    for farg, (base, stars, cname) in zip(fi["args"], params):
        assert farg in fi["decl"], f"{name}: {farg} not declared"
        ftype, attrs, dim = fi["decl"][farg]
        byval = "value" in attrs
        where = f"{name}({cname} -> {farg})"
        if stars == 0:
            assert byval, f"{where}: a C scalar is passed by value"
            assert ftype == SCALAR_KIND[base], where
            assert not dim, where
        elif stars == 1 and byval:
            assert ftype == "type(C_PTR)", f"{where}: a pointer by value is a C_PTR"
        elif stars == 1:
            if base in SCALAR_KIND:
                assert ftype == SCALAR_KIND[base], where
            elif base in STRUCTS:
                assert ftype == f"type({base})", where
            else:
                pytest.fail(f"{where}: {base} * must be a C_PTR passed by value")
        else:
            assert stars == 2, where
            assert not byval and ftype == "type(C_PTR)", f"{where}: a pointer to pointers is a C_PTR by reference"


@pytest.mark.parametrize("name", STRUCTS)
def test_derived_type_matches_struct(name):
    cs, ft = c_structs()[name], f_types()[name]
    assert [f[0] for f in cs] == [f[0] for f in ft]
    for (nm, cbase, cdim), (_, ftype, fdim) in zip(cs, ft):
        want = "type(C_PTR)" if cbase == "ptr" else SCALAR_KIND[cbase]
        assert ftype == want, f"{name}%{nm}"
        assert cdim == fdim, f"{name}%{nm}"


def test_nullable_host_arrays_are_optional():
    """mono, lin, mn, mx and ilmc's rounds may be NULL in C: optional dummies
    reach C as NULL when absent."""
    f = f_interfaces()
    for fn, args in (("adzc_tricub", ("mono", "lin", "mn", "mx")), ("adzc_tricub_sets", ("mono",)),
                     ("adzc_step_noalloc", ("mono",)), ("adzc_ilmc", ("rounds",))):
        for a in args:
            assert "optional" in f[fn]["decl"][a][1], f"{fn}({a})"


def _header_constants():
    """#define ADZC_* of the header with their values (integer or real)."""
    out = {}
    for m in re.finditer(r"^#define\s+(ADZC_\w+)\s+(.+?)\s*(?:/\*.*)?$", open(HDR).read(), re.M):
        expr = m.group(2).strip()
        shift = re.fullmatch(r"\((\d+)u?\s*<<\s*(\d+)\)", expr)
        if shift:
            out[m.group(1)] = int(shift.group(1)) << int(shift.group(2))
        elif re.fullmatch(r"-?\d+", expr):
            out[m.group(1)] = int(expr)
        elif re.fullmatch(r"-?\d+\.\d*", expr):
            out[m.group(1)] = float(expr)
    return out


def _include_parameters():
    """parameter :: NAME = value of the include, continuation lines joined."""
    text = re.sub(r"&\s*\n\s*&?", " ", open(INC).read())
    out = {}
    for m in re.finditer(r"^\s*(integer|real)\((C_\w+)\),\s*parameter\s*::\s*(.+)$", text, re.M | re.I):
        for item in m.group(3).split(","):
            name, value = (x.strip() for x in item.split("=", 1))
            value = re.sub(r"_C_\w+$", "", value)
            out[name] = float(value.replace("d", "e")) if m.group(1).lower() == "real" else int(value)
    return out


def test_constants_match_header():
    """Every ADZC_ constant of the header is a parameter of the include, with
    the same value (status codes, precisions, sets, limits)."""
    h, f = _header_constants(), _include_parameters()
    assert len(h) > 30
    missing = sorted(set(h) - set(f))
    assert not missing, missing
    assert {k: f[k] for k in h} == h
