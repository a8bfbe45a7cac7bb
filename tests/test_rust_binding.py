"""The Rust host crate (pencil-rs_b200/rust) without a Rust toolchain: its raw
FFI (src/sys.rs) is the generator's output for the current header, every C-ABI
function is declared there with the header's parameter list, and every FFI
call of the safe wrapper (src/lib.rs, examples/) names a declared function
with as many arguments as it declares."""

import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CRATE = os.path.join(ROOT, "pencil-rs_b200", "rust")
HEADER = os.path.join(ROOT, "include", "pencil_b200.h")

sys.path.insert(0, CRATE)
import gen_sys  # noqa: E402


def header_functions():
    text = gen_sys.strip_comments(open(HEADER).read())
    text = re.sub(r"^\s*#.*$", " ", text, flags=re.M)
    out = {}
    for m in re.finditer(r"\b(pb_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    return out


def rust_declarations(src):
    out = {}
    for m in re.finditer(r"pub fn (pb_\w+)\((.*?)\)( -> [^;]+)?;", src):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if not params else len(params.split(","))
    return out


def call_arg_counts(src):
    """(name, argument count) of every sys::pb_*(...) call in Rust source."""
    calls = []
    for m in re.finditer(r"sys::(pb_\w+)\(", src):
        i, depth, args, cur = m.end(), 1, [], ""
        while depth:
            c = src[i]
            if c in "([{":
                depth += 1
            elif c in ")]}":
                depth -= 1
            if depth == 1 and c == ",":
                args.append(cur)
                cur = ""
            elif depth:
                cur += c
            i += 1
        if cur.strip():
            args.append(cur)
        calls.append((m.group(1), len([a for a in args if a.strip()])))
    return calls


def test_sys_rs_is_the_generated_ffi_of_the_header():
    rc = subprocess.run([sys.executable, os.path.join(CRATE, "gen_sys.py"), "--check"]).returncode
    assert rc == 0, "src/sys.rs is stale: rerun pencil-rs_b200/rust/gen_sys.py"


def test_every_header_function_is_declared_with_its_parameters():
    hdr = header_functions()
    decl = rust_declarations(open(os.path.join(CRATE, "src", "sys.rs")).read())
    assert len(hdr) >= 60
    assert hdr == decl


def test_pointer_qualifiers_map_level_by_level():
    assert gen_sys.rust_type("pb_plan* const*") == "*const *mut pb_plan"
    assert gen_sys.rust_type("void* const*") == "*const *mut c_void"
    assert gen_sys.rust_type("const pb_geom*") == "*const pb_geom"
    assert gen_sys.rust_type("pb_plan**") == "*mut *mut pb_plan"
    assert gen_sys.rust_type("const char*") == "*const c_char"
    assert gen_sys.rust_type("int32_t") == "i32"


def test_wrapper_calls_match_the_declarations():
    decl = rust_declarations(open(os.path.join(CRATE, "src", "sys.rs")).read())
    sources = [os.path.join(CRATE, "src", "lib.rs")] + [
        os.path.join(CRATE, "examples", f) for f in os.listdir(os.path.join(CRATE, "examples"))]
    seen = set()
    for path in sources:
        src = open(path).read()
        for depth_char in "([{":
            close = {"(": ")", "[": "]", "{": "}"}[depth_char]
            assert src.count(depth_char) == src.count(close), (path, depth_char)
        for name, n in call_arg_counts(src):
            assert name in decl, (path, name)
            assert n == decl[name], (path, name, n, decl[name])
            seen.add(name)
    # the plan, transpose, remap and field entry points are all wrapped
    for name in ("pb_plan_create_c2c", "pb_plan_create_r2c", "pb_plan_create_c2r", "pb_plan_create_r2r",
                 "pb_plan_create_mixed_c2c", "pb_execute", "pb_execute_status", "pb_execute_timed",
                 "pb_transpose_create_alltoallv", "pb_transpose_create_local", "pb_transpose_execute",
                 "pb_transpose_execute_in_place", "pb_remap_create", "pb_remap_apply", "pb_field_write",
                 "pb_field_read", "pb_spectral_multiply", "pb_plan_autotune"):
        assert name in seen, name


def test_crate_manifest_pins_the_2021_edition_and_links_the_library():
    toml = open(os.path.join(CRATE, "Cargo.toml")).read()
    assert 'edition = "2021"' in toml  # extern "C" blocks without `unsafe`
    build = open(os.path.join(CRATE, "build.rs")).read()
    assert "rustc-link-lib=dylib=pencil_b200" in build
