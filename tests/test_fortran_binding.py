"""The ISO_C_BINDING module (pp-es-dg-mhd_b200/fortran/mhd_gpu_bind.f90) against the C header
(include/mhd_gpu.h), by parsing both (CPU; no Fortran compiler exists on this machine).

Checked: the same functions in the same order with the same argument counts; every by-value C
scalar is a Fortran `value` argument of the matching interoperable kind; every C pointer is either a
by-reference argument of the pointee's kind or a `type(c_ptr), value`; return types; the fields of
every struct in order; and the value of every MHD_* constant.
"""
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "mhd_gpu.h")
MODULE = os.path.join(ROOT, "pp-es-dg-mhd_b200", "fortran", "mhd_gpu_bind.f90")

C_KIND = {"int": "integer(c_int)", "double": "real(c_double)", "float": "real(c_float)",
          "long long": "integer(c_long_long)", "size_t": "integer(c_size_t)"}
OPAQUE = {"mhd_gpu_t", "mhd_batch_t", "mhd_server_t", "void"}
STRUCTS = {"mhd_gpu_status", "mhd_log_entry", "mhd_request", "mhd_request_result", "mhd_server_stats"}


def _c_source():
    return re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)


def c_functions():
    out = []
    for m in re.finditer(r"\n\s*((?:const\s+)?\w+\s*\*?)\s*(mhd_\w+)\s*\(([^)]*)\)\s*;", _c_source()):
        params = []
        for a in m.group(3).split(","):
            a = " ".join(a.replace("const ", "").split())
            stars = a.count("*")
            base = a.replace("*", " ").split()[:-1]
            params.append((" ".join(base), stars))
        out.append((m.group(2), " ".join(m.group(1).replace("const ", "").split()), params))
    return out


def c_structs():
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\}\s*\w+\s*;", _c_source(), flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.replace("const ", "").split())
            if not decl:
                continue
            names = decl.split(None, 1)[1] if not decl.startswith("long long") else decl[len("long long"):]
            for nm in names.split(","):
                nm = nm.replace("*", "").strip()
                fields.append(re.sub(r"\[\d+\]", "", nm))
        out[m.group(1)] = fields
    return out


def c_constants():
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (MHD_\w+) (-?\d+)\b", _c_source())}


def _fortran_source():
    lines = []
    for ln in open(MODULE):
        ln = ln.split("!")[0].rstrip()
        if lines and lines[-1].endswith("&"):
            lines[-1] = lines[-1][:-1] + " " + ln.strip().lstrip("&")
        else:
            lines.append(ln)
    return [l for l in lines if l.strip()]


def f_functions():
    out, cur = [], None
    for ln in _fortran_source():
        s = ln.strip()
        m = re.match(r"(integer\(c_int\)|type\(c_ptr\)) function (\w+)\(([^)]*)\)\s*bind\(C, name=\"(\w+)\"\)", s)
        if m:
            args = [a.strip() for a in m.group(3).split(",") if a.strip()]
            cur = dict(ret=m.group(1), name=m.group(2), cname=m.group(4), args=args, decl={})
            continue
        if cur is not None and s.startswith("end function"):
            out.append(cur)
            cur = None
            continue
        if cur is not None and "::" in s and not s.startswith("import"):
            attrs, names = s.split("::")
            attrs = [a.strip() for a in attrs.split(",")]
            for nm in names.split(","):
                nm = nm.strip()
                arr = nm.endswith("(*)")
                cur["decl"][nm.replace("(*)", "").strip()] = (attrs[0], "value" in attrs, arr)
    return out


def f_types():
    out, cur = {}, None
    for ln in _fortran_source():
        s = ln.strip()
        m = re.match(r"type, bind\(C\) :: (\w+)", s)
        if m:
            cur = m.group(1)
            out[cur] = []
            continue
        if cur and s.startswith("end type"):
            cur = None
            continue
        if cur and "::" in s:
            for nm in s.split("::")[1].split(","):
                out[cur].append(re.sub(r"\(\d+\)", "", nm.strip()))
    return out


def f_constants():
    out = {}
    for ln in _fortran_source():
        if "parameter ::" in ln:
            for item in ln.split("::")[1].split(","):
                k, v = item.split("=")
                out[k.strip()] = int(v.strip())
    return out


def test_same_functions_in_the_same_order():
    cf = [f[0] for f in c_functions()]
    ff = [f["cname"] for f in f_functions()]
    assert len(cf) >= 45
    assert ff == cf
    assert all(f["name"] == f["cname"] for f in f_functions())


def test_argument_counts_kinds_and_value_attributes():
    ff = {f["cname"]: f for f in f_functions()}
    for name, ret, params in c_functions():
        f = ff[name]
        assert len(f["args"]) == len(params), name
        assert f["ret"] == ("type(c_ptr)" if ret == "char *" or "*" in ret else "integer(c_int)"), name
        for arg, (base, stars) in zip(f["args"], params):
            kind, by_value, _ = f["decl"][arg]
            where = f"{name}({arg})"
            if stars == 0:  # a scalar passed by value
                assert by_value and kind == C_KIND[base], where
            elif base in OPAQUE and stars == 1:  # a handle or stream: the address itself, by value
                assert by_value and kind == "type(c_ptr)", where
            elif by_value:  # an address carried as type(c_ptr), value
                assert kind == "type(c_ptr)", where
            elif stars == 2:  # T** out-parameter: the address comes back
                assert kind == "type(c_ptr)", where
            elif base in STRUCTS:
                assert kind == f"type({base})", where
            else:
                assert kind == C_KIND[base], where


def test_struct_fields_match():
    cs, fs = c_structs(), f_types()
    assert set(cs) == set(fs) == STRUCTS
    for name in STRUCTS:
        assert fs[name] == cs[name], name


def test_constants_match():
    cc, fc = c_constants(), f_constants()
    assert len(cc) >= 25
    for k, v in cc.items():
        assert fc.get(k) == v, k
