"""The Julia binding's structs match the C ABI's field for field.

julia/FRForgeCUDA.jl declares isbits mirrors of frg_bc, frg_operators,
frg_metrics2d, frg_solve_desc and frg_result (each preceded by a
`# C: <typedef>` line).  Julia lays such structs out as the platform's C
compiler does (each field at the next multiple of its alignment, the size
rounded up to the largest alignment).  This test parses the Julia
declarations, computes every field's offset and each struct's size under
those rules, and compiles a C file of static assertions against
include/frforge_cuda.h with gcc: a field in the wrong order, of the wrong
width or missing fails the build.  No Julia and no GPU are needed.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "julia", "FRForgeCUDA.jl")

PRIM = {"Cint": (4, 4), "Int64": (8, 8), "Float64": (8, 8), "UInt8": (1, 1), "Csize_t": (8, 8)}


def parse_structs(text):
    """{julia name: (c typedef, [(field, type)])} of the `# C:` structs."""
    out = {}
    for m in re.finditer(r"#\s*C:\s*(\w+)\s*\n\s*struct\s+(\w+)\s*\n(.*?)\n\s*end\b", text, re.S):
        cname, jname, body = m.group(1), m.group(2), m.group(3)
        fields = []
        for line in body.splitlines():
            line = line.split("#")[0].strip()
            if not line:
                continue
            f = re.fullmatch(r"(\w+)::(.+)", line)
            assert f, f"cannot parse field line {line!r} of {jname}"
            fields.append((f.group(1), f.group(2).strip()))
        out[jname] = (cname, fields)
    return out


def size_align(t, structs, cache):
    if t in PRIM:
        return PRIM[t]
    if t.startswith("Ptr{"):
        return (8, 8)
    m = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", t)
    if m:
        s, a = size_align(m.group(2), structs, cache)
        return (int(m.group(1)) * s, a)
    if t in structs:
        return layout(t, structs, cache)[0:2]
    raise AssertionError(f"unknown field type {t}")


def layout(jname, structs, cache):
    """(size, align, [(field, offset)]) of a Julia isbits struct, C rules."""
    if jname in cache:
        return cache[jname]
    off, amax, offs = 0, 1, []
    for name, t in structs[jname][1]:
        s, a = size_align(t, structs, cache)
        off = (off + a - 1) // a * a
        offs.append((name, off))
        off += s
        amax = max(amax, a)
    size = (off + amax - 1) // amax * amax
    cache[jname] = (size, amax, offs)
    return cache[jname]


def test_shim_declares_the_abi_structs():
    with open(SHIM) as f:
        structs = parse_structs(f.read())
    assert {c for c, _ in structs.values()} == {"frg_bc", "frg_operators", "frg_metrics2d", "frg_solve_desc",
                                                 "frg_result"}


def test_shim_layout_matches_header(tmp_path):
    with open(SHIM) as f:
        structs = parse_structs(f.read())
    cache = {}
    lines = ['#include <stddef.h>', '#include "frforge_cuda.h"']
    n = 0
    for jname, (cname, _) in structs.items():
        size, _, offs = layout(jname, structs, cache)
        lines.append(f'_Static_assert(sizeof({cname}) == {size}, "sizeof {cname}: Julia {jname} is {size}");')
        for field, off in offs:
            lines.append(f'_Static_assert(offsetof({cname}, {field}) == {off}, '
                         f'"{cname}.{field}: Julia {jname} puts it at {off}");')
            n += 1
    src = tmp_path / "layout_check.c"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert n >= 60  # every field of the five structs was checked


def test_layout_check_catches_a_swapped_field(tmp_path):
    # the check itself: two fields swapped in a copy of the declarations fail it
    with open(SHIM) as f:
        text = f.read()
    bad = text.replace("    nx::Cint\n    ny::Cint\n    x_left::Float64", "    nx::Cint\n    x_left::Float64\n"
                       "    ny::Cint", 1)
    assert bad != text
    structs = parse_structs(bad)
    size, _, offs = layout("FrgSolveDesc", structs, {})
    lines = ['#include <stddef.h>', '#include "frforge_cuda.h"']
    lines += [f"_Static_assert(offsetof(frg_solve_desc, {fd}) == {o}, \"{fd}\");" for fd, o in offs]
    src = tmp_path / "bad.c"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode != 0
