"""CPU: the Fortran binding (pepc_b200/fortran/module_pepcg.f90) against the C
header it binds (include/pepcg.h).  No Fortran compiler is needed: the test
reads both sources and checks that

  * the bind(c) derived type pepcg_params lists the C struct's fields in the
    same order, with the same kinds and array lengths (a drift here makes a
    Fortran caller write one field through another's bytes);
  * every bind(c, name=...) interface names a function that the header
    declares, with the same number of arguments."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pepcg.h")
FORTRAN = os.path.join(ROOT, "pepc_b200", "fortran", "module_pepcg.f90")

C_KIND = {"double": "c_double", "int32_t": "c_int32_t", "int64_t": "c_int64_t"}


def c_struct_fields(name):
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\}\s*%s;" % (name, name), txt, flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ctype, rest = decl.split(None, 1)
        for item in rest.split(","):
            m = re.fullmatch(r"\s*(\w+)\s*(?:\[(\d+)\])?\s*", item)
            out.append((C_KIND[ctype], m.group(1), int(m.group(2) or 1)))
    return out


def fortran_type_fields(name):
    src = open(FORTRAN).read()
    body = re.search(r"type, bind\(c\), public :: %s\n(.*?)\n\s*end type" % name, src,
                     flags=re.S).group(1)
    out = []
    for line in body.splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        m = re.fullmatch(r"(real|integer)\((c_\w+)\)\s*::\s*(.*)", line)
        assert m, line
        for item in re.findall(r"\w+(?:\(\d+\))?", m.group(3)):
            mm = re.fullmatch(r"(\w+)(?:\((\d+)\))?", item)
            out.append((m.group(2), mm.group(1), int(mm.group(2) or 1)))
    return out


def test_params_type_matches_header_field_by_field():
    c = c_struct_fields("pepcg_params")
    f = fortran_type_fields("pepcg_params")
    assert f == c


def c_functions():
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|void|const char\*|int64_t|long long)\s+\**(pepcg_\w+)\s*\(([^)]*)\)",
                         txt):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def fortran_interfaces():
    src = open(FORTRAN).read()
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+\w+\s*\(([^)]*)\)\s*&?\s*bind\(c, name=\"(\w+)\"\)",
                         src, flags=re.S):
        args = [a for a in m.group(1).replace("&", " ").split(",") if a.strip()]
        out[m.group(2)] = len(args)
    return out


def test_interfaces_bind_declared_functions():
    c = c_functions()
    f = fortran_interfaces()
    assert {"pepcg_create", "pepcg_grow_tree", "pepcg_traverse_tree", "pepcg_sort_keys",
            "pepcg_lattice_force"} <= set(f)
    for name, nargs in f.items():
        assert name in c, name
        assert c[name] == nargs, (name, nargs, c[name])
