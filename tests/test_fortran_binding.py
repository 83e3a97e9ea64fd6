"""The Fortran binding (include/module_gpu.f90) against the C header it binds.

No Fortran compiler exists here, so the layout a `bind(C)` derived type gets is
derived from the module text with the rules the Fortran standard gives such
types (the companion C compiler's layout: c_int 4 bytes, c_double 8 bytes, each
aligned to its size) and compared with the offsets and sizes gcc reports for
`hc_params` and `hc_diag` when it compiles include/hercules_b200.h, and with
the ctypes images the Python host uses. Every entry point the header declares
must be bound in the module under its own name with the same argument count.
"""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from hercules_b200.params import HcDiag, HcParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "module_gpu.f90")
HDR = os.path.join(ROOT, "include", "hercules_b200.h")
KIND = {"integer(c_int)": (4, 4), "real(c_double)": (8, 8)}


def _strip_comments(text):
    return "\n".join(line.split("!")[0] for line in text.splitlines())


def fortran_types():
    """{type name: [(member, kind, count)]} of the bind(C) types, in order."""
    text = _strip_comments(open(F90).read())
    out = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", text, re.S | re.I):
        members = []
        for line in m.group(2).splitlines():
            d = re.match(r"\s*(integer\(c_int\)|real\(c_double\))\s*::\s*(.+)", line, re.I)
            if not d:
                continue
            for item in d.group(2).split(","):
                item = item.strip()
                a = re.match(r"(\w+)(?:\((\d+)\))?$", item)
                members.append((a.group(1), d.group(1).lower(), int(a.group(2) or 1)))
        out[m.group(1).lower()] = members
    return out


def c_layout(members):
    """Offsets and size under the C rules for bind(C) types."""
    off, align, res = 0, 1, {}
    for name, kind, count in members:
        size, al = KIND[kind]
        off = (off + al - 1) // al * al
        res[name] = off
        off += size * count
        align = max(align, al)
    return res, (off + align - 1) // align * align


def gcc_layout(struct, members):
    src = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HDR}"', "int main(void) {"]
    for name, _, _ in members:
        src.append(f'  printf("{name} %zu\\n", offsetof({struct}, {name}));')
    src.append(f'  printf("__size__ %zu\\n", sizeof({struct}));')
    src.append("  return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(c, "w").write("\n".join(src))
        subprocess.check_call(["gcc", "-std=c99", "-Wall", "-o", exe, c])
        out = subprocess.check_output([exe]).decode()
    vals = dict(line.split() for line in out.splitlines())
    return {k: int(v) for k, v in vals.items() if k != "__size__"}, int(vals["__size__"])


@pytest.mark.parametrize("struct,ctype", [("hc_params", HcParams), ("hc_diag", HcDiag)])
def test_bind_c_types_match_the_header(struct, ctype):
    members = fortran_types()[struct]
    f_off, f_size = c_layout(members)
    g_off, g_size = gcc_layout(struct, members)
    assert f_off == g_off
    assert f_size == g_size
    # the ctypes image used by the Python host has the same layout
    assert ctypes.sizeof(ctype) == g_size
    for name, _ in ctype._fields_:
        assert getattr(ctype, name).offset == g_off[name], name


def header_prototypes():
    txt = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(hc_[a-z_]+)\s*\(([^;{]*?)\)\s*;", txt, re.S):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def fortran_interfaces():
    text = _strip_comments(open(F90).read()).replace("&\n", " ")
    out = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", text, re.I):
        args = [a for a in m.group(2).split(",") if a.strip()]
        assert m.group(1) == m.group(3)
        out[m.group(3)] = len(args)
    return out


def test_every_entry_point_is_bound_with_its_arity():
    hdr, f90 = header_prototypes(), fortran_interfaces()
    assert sorted(hdr) == sorted(f90)
    for name, n in hdr.items():
        assert f90[name] == n, name
