"""The Fortran binding include/pibm.f90 against the C header include/pibm.h.

No Fortran compiler is available, so the module is checked by reading it:

* every bind(C) derived type is laid out with the C rules that bind(C)
  guarantees (each member at the next multiple of its alignment, the size
  rounded up to the largest alignment) and every member offset and the size
  are compared with offsetof / sizeof of the C struct of the same name,
  printed by a program that gcc compiles against the header;
* the set of bind(C) interfaces equals the set of entry points the header
  declares, with the same number of arguments each, and the shared library
  exports every one of them.
"""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "pibm.f90")
HDR = os.path.join(ROOT, "include", "pibm.h")

_KIND = {"c_int32_t": 4, "c_int": 4, "c_int64_t": 8, "c_long_long": 8, "c_double": 8, "c_int8_t": 1}


def _fortran_types():
    """{type name: [(member, size, align, count)]} of every bind(C) type."""
    text = open(F90).read()
    out = {}
    for m in re.finditer(r"type\s*,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", text, flags=re.S | re.I):
        members = []
        for line in m.group(2).splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            d = re.match(r"(integer|real|type)\((\w+)\)\s*::\s*(.*)", line, flags=re.I)
            assert d, line
            base, kind, names = d.group(1).lower(), d.group(2).lower(), d.group(3)
            size = 8 if (base == "type" and kind == "c_ptr") else _KIND[kind]
            for nm in re.finditer(r"(\w+)(?:\((\d+)\))?", names):
                members.append((nm.group(1), size, size, int(nm.group(2) or 1)))
        out[m.group(1).lower()] = members
    return out


def _c_layout(members):
    off, offs, amax = 0, [], 1
    for name, size, align, count in members:
        off = (off + align - 1) // align * align
        offs.append((name, off))
        off += size * count
        amax = max(amax, align)
    return offs, (off + amax - 1) // amax * amax


def _header_offsets(types, tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "pibm.h"', "int main(void) {"]
    for t, members in types.items():
        lines.append(f'printf("{t} sizeof %zu\\n", sizeof({t}));')
        for name, *_ in members:
            lines.append(f'printf("{t} {name} %zu\\n", offsetof({t}, {name}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for row in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n"):
        if row:
            t, name, v = row.split()
            got[(t, name)] = int(v)
    return got


def test_bind_c_types_match_the_header(tmp_path):
    types = _fortran_types()
    assert set(types) == {"pibm_params", "pibm_particles", "pibm_state_view", "pibm_step_report", "pibm_info",
                          "pibm_adjoint_report"}
    c = _header_offsets(types, tmp_path)
    for t, members in types.items():
        offs, size = _c_layout(members)
        for name, off in offs:
            assert c[(t, name)] == off, (t, name, off, c[(t, name)])
        assert c[(t, "sizeof")] == size, (t, size, c[(t, "sizeof")])


def _header_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"^[\w\s\*]*?\b(pibm_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.M | re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def _fortran_functions():
    text = open(F90).read()
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*(?:&\s*\n\s*)?bind\(C,\s*name=\"(\w+)\"\)",
                         text, flags=re.I):
        args = m.group(2).strip()
        assert m.group(1) == m.group(3)
        out[m.group(3)] = 0 if not args else args.count(",") + 1
    return out


def test_interfaces_match_the_header():
    h, f = _header_functions(), _fortran_functions()
    assert "pibm_create" in h and "pibm_batch_destroy" in h
    assert set(f) == set(h), (set(h) - set(f), set(f) - set(h))
    for name, n in h.items():
        assert f[name] == n, (name, n, f[name])


def test_library_exports_every_interface():
    lib_path = os.path.join(ROOT, "pureibm_ps2d_fd1d_b200", "_lib", "libpibm.so")
    if not os.path.exists(lib_path):
        pytest.skip("libpibm.so is not built")
    lib = ctypes.CDLL(lib_path)
    for name in _fortran_functions():
        assert hasattr(lib, name), name
