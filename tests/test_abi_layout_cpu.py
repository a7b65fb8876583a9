"""The struct layouts of the C ABI agree in all three places a host reads them.

include/shygpu.h declares the structs the library reads; shygpu/abi.py (and
shygpu.ZetaSystem) mirror them for ctypes; INTEGRATION.md gives the Fortran
`bind(C)` types a SHYFEM host would compile.  A field added, moved or retyped
in one of them and not the others would make the library read a different
record than the host wrote, so this test parses all three and compares field
names, order and types, and compares ctypes' sizes and offsets with the ones
gcc computes from the header.
"""
import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import pytest

import shygpu
from shygpu import abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "shygpu.h"
INTEGRATION = ROOT / "INTEGRATION.md"

# header struct -> (ctypes mirror, Fortran type name in INTEGRATION.md)
STRUCTS = {
    "shy_basin": (abi.ShyBasin, "shy_basin"),
    "shy_params": (abi.ShyParams, "shy_params"),
    "shy_state": (abi.ShyState, "shy_state"),
    "shy_step_info": (abi.ShyStepInfo, "shy_step_info"),
    "shy_zeta_system_t": (shygpu.ZetaSystem, "shy_zeta_system_t"),
}

C_TYPES = {"int32_t": "i32", "float": "f32", "double": "f64"}
F_TYPES = {"integer(c_int32_t)": "i32", "real(c_float)": "f32", "real(c_double)": "f64",
           "type(c_ptr)": "ptr"}


def header_structs():
    """{name: [(field, kind, count)]} from the typedef structs of the header."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", text, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            dm = re.match(r"(?:const\s+)?(\w+)\s+(.*)$", decl, flags=re.S)
            base, rest = dm.group(1), dm.group(2)
            for d in rest.split(","):
                fm = re.match(r"\s*(\*?)\s*(\w+)\s*(?:\[(\d+)\])?\s*$", d)
                assert fm, f"unparsed declarator {d!r} in {m.group(1)}"
                kind = "ptr" if fm.group(1) else C_TYPES[base]
                fields.append((fm.group(2), kind, int(fm.group(3) or 1)))
        out[m.group(1)] = fields
    return out


def ctypes_fields(cls):
    fields = []
    for name, t in cls._fields_:
        count = 1
        if issubclass(t, C.Array):
            count, t = t._length_, t._type_
        if issubclass(t, (C._Pointer, C.c_void_p)):
            kind = "ptr"
        else:
            kind = {C.c_int32: "i32", C.c_float: "f32", C.c_double: "f64"}[t]
        fields.append((name, kind, count))
    return fields


def fortran_types():
    """{name: [(field, kind, count)]} from the `type, bind(C)` blocks of
    INTEGRATION.md's code listings."""
    out = {}
    text = INTEGRATION.read_text()
    for m in re.finditer(r"type, bind\(C\) :: (\w+)\n(.*?)\n\s*end type", text, flags=re.S):
        fields = []
        for line in m.group(2).splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            tm = re.match(r"(\w+\(\w+\))\s*::\s*(.*)$", line)
            assert tm, f"unparsed line {line!r} in {m.group(1)}"
            kind = F_TYPES[tm.group(1)]
            for v in re.findall(r"(\w+)(?:\(([\d,]+)\))?", tm.group(2)):
                count = 1
                for d in (v[1].split(",") if v[1] else []):
                    count *= int(d)
                fields.append((v[0], kind, count))
        out[m.group(1)] = fields
    return out


def test_header_and_ctypes_mirror_agree():
    hs = header_structs()
    for name, (cls, _) in STRUCTS.items():
        assert name in hs, name
        assert ctypes_fields(cls) == hs[name], name


def test_header_and_fortran_binding_agree():
    hs = header_structs()
    fs = fortran_types()
    for name, (_, fname) in STRUCTS.items():
        assert fname in fs, f"INTEGRATION.md declares no bind(C) type {fname}"
        assert fs[fname] == hs[name], name


def test_every_header_struct_is_mirrored():
    assert set(header_structs()) == set(STRUCTS)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_sizes_and_offsets_match_the_c_compiler(tmp_path):
    """gcc's sizeof/offsetof of each header struct equal ctypes'."""
    hs = header_structs()
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "shygpu.h"', "int main(void) {"]
    for name, fields in hs.items():
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for f, _, _ in fields:
            lines.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for name, (cls, _) in STRUCTS.items():
        assert got[(name, "sizeof")] == C.sizeof(cls), name
        for f, _, _ in hs[name]:
            assert got[(name, f)] == getattr(cls, f).offset, (name, f)
