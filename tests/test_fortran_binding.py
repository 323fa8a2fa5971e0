"""The Fortran interface module of INTEGRATION.md against include/tis_b200.h.

No Fortran compiler exists on this machine, so the module is checked as
text: its bind(C) derived types must list the C structs' fields in the same
order with the same kinds (int32_t <-> c_int32_t, 64-bit integers <->
c_int64_t, double <-> c_double, pointers <-> c_ptr, the same array
lengths), every entry point of the header must have a bind(C) interface,
and each interface must take as many arguments as the C prototype.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header():
    src = open(os.path.join(ROOT, "include", "tis_b200.h")).read()
    return re.sub(r"/\*.*?\*/", " ", src, flags=re.S)


def fortran_module():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```fortran\n(.*?)```", text, flags=re.S)
    assert m, "no fortran block"
    lines = []
    for line in m.group(1).split("\n"):
        line = line.split("!")[0].rstrip()
        if lines and lines[-1].endswith("&"):
            lines[-1] = lines[-1][:-1] + " " + line.strip()
        else:
            lines.append(line)
    return lines


def c_struct_fields(name):
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), header(), flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"(const )?(int32_t|uint64_t|int64_t|double|char) (.*)", decl)
        assert m, decl
        base = m.group(2)
        for d in m.group(3).split(","):
            d = d.strip()
            ptr = d.startswith("*")
            d = d.lstrip("*").strip()
            arr = re.match(r"(\w+)\[(\d+)\]", d)
            nm, n = (arr.group(1), int(arr.group(2))) if arr else (d, 1)
            kind = "c_ptr" if ptr else {"int32_t": "c_int32_t", "uint64_t": "c_int64_t", "int64_t": "c_int64_t",
                                        "double": "c_double"}[base]
            out.append((nm.lower(), kind, n))
    return out


def f_type_fields(name):
    lines = fortran_module()
    start = next(i for i, l in enumerate(lines) if re.match(r"\s*type, bind\(C\) :: %s\s*$" % name, l))
    out = []
    for line in lines[start + 1:]:
        if re.match(r"\s*end type", line):
            break
        if "::" not in line:
            continue
        spec, names = line.split("::")
        kind = re.search(r"\((c_\w+)\)", spec).group(1)
        for d in re.findall(r"\w+(?:\(\d+\))?", names):
            arr = re.match(r"(\w+)\((\d+)\)", d)
            nm, n = (arr.group(1), int(arr.group(2))) if arr else (d, 1)
            out.append((nm.lower(), kind, n))
    return out


@pytest.mark.parametrize("cname,fname", [("tis_topology", "tis_topology"), ("tis_params", "tis_params"),
                                         ("tis_status_t", "tis_status_t")])
def test_derived_types_match_the_c_structs(cname, fname):
    assert f_type_fields(fname) == c_struct_fields(cname)


def c_prototypes():
    protos = {}
    for m in re.finditer(r"^[\w ]+?\*?\s*(tis_\w+)\(([^)]*)\);", header(), flags=re.M):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        protos[m.group(1)] = len(args)
    return protos


def f_interfaces():
    out = {}
    for line in fortran_module():
        m = re.search(r"(?:function|subroutine) (\w+)\(([^)]*)\)\s*(?:&\s*)?bind\(C, name=\"(tis_\w+)\"\)", line)
        if m:
            args = [a for a in m.group(2).split(",") if a.strip()]
            out[m.group(3)] = len(args)
    return out


def test_every_entry_point_has_an_interface_with_its_arguments():
    protos, ifaces = c_prototypes(), f_interfaces()
    assert len(protos) > 30
    missing = sorted(set(protos) - set(ifaces))
    assert not missing, missing
    for name, n in ifaces.items():
        assert name in protos, name
        assert n == protos[name], (name, n, protos[name])
