"""The Rust `-sys` crate's bindings (include/rust/exg-cuda-sys), checked without a Rust toolchain:
the committed src/lib.rs is what include/rust/gen_ffi.py makes from include/exg.h, it binds every
EXG_API entry point with its parameter count, and each #[repr(C)] struct lays out its fields at the
offsets the C compiler gives the header's struct (repr(C) follows the C rules, computed here from
the Rust field types)."""
import importlib.util
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(ROOT, "include", "rust", "gen_ffi.py")
LIB_RS = os.path.join(ROOT, "include", "rust", "exg-cuda-sys", "src", "lib.rs")


def gen():
    spec = importlib.util.spec_from_file_location("gen_ffi", GEN)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_committed_bindings_are_current():
    with open(LIB_RS) as f:
        assert f.read() == gen().generate(), "run python include/rust/gen_ffi.py"


def test_every_entry_point_is_bound():
    g = gen()
    with open(g.HEADER) as f:
        consts, structs, handles, funcs = g.parse(f.read())
    with open(g.HEADER) as f:
        declared = re.findall(r"EXG_API\s+[\w\s\*]*?\b(exg_\w+)\s*\(", g.strip_comments(f.read()))
    assert len(declared) == len(funcs) > 0 and sorted(declared) == sorted(f[0] for f in funcs)
    with open(LIB_RS) as f:
        rs = f.read()
    for name, _, params in funcs:
        m = re.search(r"pub fn " + name + r"\((.*?)\)", rs)
        assert m, name
        n = 0 if not m.group(1).strip() else m.group(1).count(":")
        assert n == len(params), name


def c_offsets(structs):
    """sizeof and offsetof of every field, from gcc compiling the header."""
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "exg.h"', "int main(void) {"]
    for name, fields in structs:
        lines.append(f'  printf("{name} %zu", sizeof({name}));')
        for fname, _, _ in fields:
            lines.append(f'  printf(" %zu", offsetof({name}, {fname}));')
        lines.append('  printf("\\n");')
    lines.append("  return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "o.c"), os.path.join(d, "o")
        with open(src, "w") as f:
            f.write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.strip().splitlines():
        parts = line.split()
        res[parts[0]] = [int(x) for x in parts[1:]]
    return res


def test_struct_layouts_match_the_c_compiler():
    g = gen()
    with open(g.HEADER) as f:
        consts, structs, handles, funcs = g.parse(f.read())
    want = c_offsets(structs)
    with open(LIB_RS) as f:
        rs = f.read()
    for name, fields in structs:
        body = re.search(r"pub struct " + name + r" \{(.*?)\n\}", rs, flags=re.S).group(1)
        off, align_max, got = 0, 1, []
        for fname, rtype in re.findall(r"pub (\w+): ([^,]+),", body):
            m = re.match(r"\[(.+); (\d+)\]$", rtype)
            elem, count = (m.group(1), int(m.group(2))) if m else (rtype, 1)
            size, align = g.RUST_LAYOUT[elem]
            off = (off + align - 1) // align * align
            got.append(off)
            off += size * count
            align_max = max(align_max, align)
        total = (off + align_max - 1) // align_max * align_max
        assert [total] + got == want[name], (name, [total] + got, want[name])
