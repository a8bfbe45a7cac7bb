"""Generates src/sys.rs, the raw Rust FFI of the C-ABI, from
include/pencil_b200.h (a bindgen stand-in for this one header; the image that
builds the library has no Rust toolchain).

Every ``#define`` constant, enum, struct (opaque or with fields) and function
prototype of the header becomes its ``#[repr(C)]`` / ``extern "C"``
counterpart with the same names and field order.  C pointer qualifiers map
onto ``*const`` / ``*mut`` level by level (``pb_plan* const* plans`` ->
``*const *mut pb_plan``).

Run from anywhere: ``python gen_sys.py`` rewrites ``src/sys.rs``;
``python gen_sys.py --check`` exits 1 if the committed file is stale.
"""

from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "pencil_b200.h")
OUT = os.path.join(HERE, "src", "sys.rs")

BASE = {"int32_t": "i32", "int64_t": "i64", "uint8_t": "u8", "int8_t": "i8", "uint32_t": "u32",
        "uint64_t": "u64", "int16_t": "i16", "uint16_t": "u16", "size_t": "usize", "int": "c_int",
        "double": "f64", "float": "f32", "char": "c_char", "void": "c_void"}


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def rust_type(ctype: str) -> str:
    """C type (no declarator name) -> Rust type."""
    toks = re.findall(r"[A-Za-z_][A-Za-z0-9_]*|\*", ctype)
    base, base_const, i = None, False, 0
    while i < len(toks) and toks[i] != "*":
        if toks[i] == "const":
            base_const = True
        elif toks[i] in ("struct", "enum", "unsigned", "signed"):
            pass
        else:
            base = toks[i]
        i += 1
    if base is None:
        raise ValueError(f"no base type in {ctype!r}")
    # levels[k] = (rust text of level k, whether level k itself is const)
    text, const = BASE.get(base, base), base_const
    while i < len(toks):
        if toks[i] == "*":
            text = ("*const " if const else "*mut ") + text
            const = False
        elif toks[i] == "const":
            const = True
        i += 1
    return text


def split_decl(decl: str):
    """'const pb_geom* geom' -> ('const pb_geom*', 'geom')."""
    decl = decl.strip()
    m = re.match(r"^(.*?)([A-Za-z_][A-Za-z0-9_]*)\s*$", decl, flags=re.S)
    if not m:
        raise ValueError(f"cannot split {decl!r}")
    return m.group(1).strip(), m.group(2)


def const_value(expr: str, defines: dict) -> str:
    e = expr.strip()
    e = re.sub(r"(\d+)[uUlL]+", r"\1", e)
    for k, v in defines.items():
        e = re.sub(rf"\b{k}\b", v, e)
    if e.startswith("(") and e.endswith(")") and e.count("(") == 1:
        e = e[1:-1].strip()
    return e


def generate(header_text: str) -> str:
    raw = header_text
    text = strip_comments(raw)
    out = ["// Generated by gen_sys.py from include/pencil_b200.h -- do not edit by hand.",
           "// Raw FFI of libpencil_b200.so (the C-ABI of the B200 pencil FFT library).",
           "#![allow(non_camel_case_types, non_upper_case_globals, dead_code, clippy::all)]",
           "",
           "use std::os::raw::{c_char, c_int, c_void};",
           ""]
    defines = {}
    # #define constants (integer expressions), in header order
    for m in re.finditer(r"^\s*#define\s+([A-Z_][A-Z0-9_]*)\s+(.+?)\s*$", text, flags=re.M):
        name, val = m.group(1), m.group(2)
        if name.endswith("_H"):
            continue
        v = const_value(val, defines)
        defines[name] = f"({v})" if re.search(r"[*+\-/ ]", v) else v
        ty = "usize" if name.endswith("_BYTES") else "i32"
        out.append(f"pub const {name}: {ty} = {v};")
    out.append("")
    body = re.sub(r"^\s*#.*$", " ", text, flags=re.M)
    body = body.replace('extern "C" {', " ")
    # enums
    for m in re.finditer(r"typedef\s+enum\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", body, flags=re.S):
        name = m.group(3)
        out.append(f"pub type {name} = c_int;")
        for item in m.group(2).split(","):
            item = item.strip()
            if not item:
                continue
            k, v = [s.strip() for s in item.split("=")]
            out.append(f"pub const {k}: {name} = {v};")
        out.append("")
    body = re.sub(r"typedef\s+enum\s+\w+\s*\{.*?\}\s*\w+\s*;", " ", body, flags=re.S)
    # structs with fields
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", body, flags=re.S):
        name = m.group(3)
        out.append("#[repr(C)]")
        out.append("#[derive(Clone, Copy, Debug, Default)]")
        out.append(f"pub struct {name} {{")
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            first = re.match(r"^([A-Za-z_][A-Za-z0-9_]*(?:\s*\*)*)\s+(.*)$", decl, flags=re.S)
            ctype, names = first.group(1), first.group(2)
            for nm in names.split(","):
                nm = nm.strip()
                arr = re.match(r"^(\w+)\s*\[\s*(\w+)\s*\]$", nm)
                if arr:
                    n = defines.get(arr.group(2), arr.group(2))
                    out.append(f"    pub {arr.group(1)}: [{rust_type(ctype)}; {n}],")
                else:
                    out.append(f"    pub {nm}: {rust_type(ctype)},")
        out.append("}")
        out.append("")
    body = re.sub(r"typedef\s+struct\s+\w+\s*\{.*?\}\s*\w+\s*;", " ", body, flags=re.S)
    # opaque handles
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s+(\w+)\s*;", body):
        out.append("#[repr(C)]")
        out.append(f"pub struct {m.group(2)} {{")
        out.append("    _private: [u8; 0],")
        out.append("}")
        out.append("")
    body = re.sub(r"typedef\s+struct\s+\w+\s+\w+\s*;", " ", body)
    # function prototypes
    out.append('#[link(name = "pencil_b200")]')
    out.append('extern "C" {')
    for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_\s\*]*?)\b(pb_\w+)\s*\(([^;]*?)\)\s*;", body, flags=re.S):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        args = []
        if params and params != "void":
            for p in params.split(","):
                ctype, pname = split_decl(" ".join(p.split()))
                if pname in ("in", "ref", "type", "mod", "fn", "move", "loop", "match"):
                    pname = pname + "_"
                args.append(f"{pname}: {rust_type(ctype)}")
        rt = rust_type(ret)
        tail = "" if rt == "c_void" else f" -> {rt}"
        out.append(f"    pub fn {name}({', '.join(args)}){tail};")
    out.append("}")
    out.append("")
    return "\n".join(out)


def main(argv):
    with open(HEADER) as f:
        src = generate(f.read())
    if "--check" in argv:
        with open(OUT) as f:
            return 0 if f.read() == src else 1
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as f:
        f.write(src)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
