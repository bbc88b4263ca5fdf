"""Generates the Rust `-sys` crate's bindings (exg-cuda-sys/src/lib.rs) from include/exg.h.

The reference's host is a Rust workspace; a maintainer binds this library from it with a `-sys`
crate in place of rembrandt's Vulkan device layer and the storage half of aristotle (the crate's
Cargo.toml and build.rs sit beside the generated file). This is what `bindgen include/exg.h`
would emit, restricted to what the header declares: integer constants (#define and enum
values), the record structs (#[repr(C)], same fields in the same order), the opaque handles and
every EXG_API entry point. No Rust toolchain is needed to run it; tests/test_rust_ffi.py checks that
the committed file is what this script makes, that it binds every entry point, and that each
struct's field offsets equal the C compiler's.

Run: python include/rust/gen_ffi.py        (rewrites exg-cuda-sys/src/lib.rs)
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "..", "exg.h")
OUT = os.path.join(HERE, "exg-cuda-sys", "src", "lib.rs")

SCALARS = {"int32_t": "i32", "int64_t": "i64", "uint32_t": "u32", "uint64_t": "u64", "double": "f64",
           "float": "f32", "size_t": "usize", "int": "c_int", "char": "c_char", "void": "c_void"}
# (size, alignment) of the Rust types the structs use, for the layout check (repr(C) = C rules)
RUST_LAYOUT = {"i32": (4, 4), "u32": (4, 4), "i64": (8, 8), "u64": (8, 8), "f64": (8, 8), "f32": (4, 4),
               "usize": (8, 8), "c_int": (4, 4), "*mut c_void": (8, 8), "*const c_void": (8, 8)}


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def parse(text):
    """(constants, structs, handles, functions) of the header text."""
    src = strip_comments(text)
    consts = []
    for name, val in re.findall(r"#define\s+(EXG_[A-Z0-9_]+)\s+(-?\d+)\b", src):
        consts.append((name, int(val)))
    for body in re.findall(r"typedef\s+enum\s*\{(.*?)\}\s*\w+\s*;", src, flags=re.S):
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            m = re.match(r"(EXG_[A-Z0-9_]+)\s*=\s*(-?\d+)$", item)
            if not m:
                raise ValueError(f"enum item without an explicit value: {item!r}")
            consts.append((m.group(1), int(m.group(2))))
    structs = []
    for body, name in re.findall(r"typedef\s+struct\s*\{(.*?)\}\s*(exg_\w+)\s*;", src, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"((?:const\s+)?[a-z_0-9]+(?:\s*\*)?)\s+(.*)$", decl)
            ctype, names = m.group(1).replace(" ", ""), m.group(2)
            for nm in names.split(","):
                nm = nm.strip()
                am = re.match(r"(\w+)\s*\[(\d+)\]$", nm)
                if am:
                    fields.append((am.group(1), ctype, int(am.group(2))))
                else:
                    fields.append((nm.lstrip("*"), ctype + ("*" if nm.startswith("*") else ""), None))
        structs.append((name, fields))
    handles = re.findall(r"typedef\s+struct\s+(exg_\w+_s)\s*\*\s*(exg_\w+_t)\s*;", src)
    funcs = []
    for ret, name, args in re.findall(r"EXG_API\s+((?:const\s+)?\w+\s*\**)\s*(exg_\w+)\s*\((.*?)\)\s*;", src,
                                      flags=re.S):
        params = []
        args = " ".join(args.split())
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                m = re.match(r"(.*?)(\w+)\s*(\[\d*\])?$", a)
                ctype = m.group(1).strip()
                if m.group(3):  # an array parameter decays to a pointer
                    ctype += "*"
                params.append((m.group(2), ctype.replace(" *", "*").replace("* ", "*")))
        funcs.append((name, ret.strip(), params))
    return consts, structs, handles, funcs


def rust_type(ctype, handles):
    ctype = " ".join(ctype.split()).replace(" *", "*")
    const = ctype.startswith("const ")
    base = ctype[6:] if const else ctype
    stars = base.count("*")
    base = base.replace("*", "").strip()
    if base in handles:
        r = base
    elif base in SCALARS:
        r = SCALARS[base]
    elif base.startswith("exg_"):
        r = base
    else:
        raise ValueError(f"unmapped C type {ctype!r}")
    for k in range(stars):
        r = ("*const " if const and k == 0 else "*mut ") + r
    return r


def emit(consts, structs, handles, funcs):
    hnames = {h for _, h in handles}
    out = ["// Generated by include/rust/gen_ffi.py from include/exg.h; do not edit by hand.",
           "//! Raw bindings of the B200 per-step dynamics library (libexg.so, include/exg.h).",
           "//! Every entry point returns an exg_status (EXG_OK = 0, negative = error); see the header",
           "//! for each call's contract.",
           "#![allow(non_camel_case_types, non_upper_case_globals, non_snake_case, dead_code)]",
           "",
           "use std::os::raw::{c_char, c_int, c_void};",
           ""]
    for name, val in consts:
        out.append(f"pub const {name}: c_int = {val};")
    out.append("")
    for sname, hname in handles:
        out.append("#[repr(C)]")
        out.append(f"pub struct {sname} {{")
        out.append("    _private: [u8; 0],")
        out.append("}")
        out.append(f"pub type {hname} = *mut {sname};")
    out.append("")
    for name, fields in structs:
        out.append("#[repr(C)]")
        out.append("#[derive(Clone, Copy, Debug)]")
        out.append(f"pub struct {name} {{")
        for fname, ctype, n in fields:
            t = rust_type(ctype, hnames)
            out.append(f"    pub {fname}: [{t}; {n}]," if n else f"    pub {fname}: {t},")
        out.append("}")
        out.append("")
    out.append('#[link(name = "exg")]')
    out.append('extern "C" {')
    for name, ret, params in funcs:
        ps = ", ".join(f"{p}: {rust_type(t, hnames)}" for p, t in params)
        r = rust_type(ret, hnames)
        tail = "" if r == "c_void" else f" -> {r}"
        out.append(f"    pub fn {name}({ps}){tail};")
    out.append("}")
    out.append("")
    return "\n".join(out)


def generate():
    with open(HEADER) as f:
        return emit(*parse(f.read()))


if __name__ == "__main__":
    text = generate()
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as f:
        f.write(text)
    print(f"wrote {OUT}", file=sys.stderr)
