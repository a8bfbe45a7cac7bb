"""The build's header dependencies: an object is rebuilt when its source or a
header that it includes, directly or through other headers, is newer.  A
header the scan misses would leave a stale object in the library."""

import os
import re
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "pencil-rs_b200"))

from pencil_b200 import _build as B  # noqa: E402

QUOTED = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _direct(path):
    with open(path) as f:
        return set(QUOTED.findall(f.read()))


def test_every_quoted_include_resolves_and_is_tracked():
    for src, _, _ in B.SOURCES:
        path = os.path.join(B.CSRC, src)
        deps = {os.path.basename(d) for d in B._includes(path)}
        assert _direct(path) <= deps, (src, _direct(path) - deps)
        # closure: what each tracked header includes is tracked too
        for d in B._includes(path):
            assert {os.path.basename(x) for x in B._includes(d)} <= deps, (src, d)


def test_kernel_headers_reach_only_their_users():
    users = {src for src, _, _ in B.SOURCES
             if "mr_bs.cuh" in {os.path.basename(d) for d in B._includes(os.path.join(B.CSRC, src))}}
    assert users == {"mr_bs_kernels.cu"}, users
    r2r = {src for src, _, _ in B.SOURCES
           if "mr_r2r.cuh" in {os.path.basename(d) for d in B._includes(os.path.join(B.CSRC, src))}}
    assert r2r == {"mr_r2r_kernels.cu"}, r2r


def test_public_header_is_a_dependency_of_the_host_code():
    deps = {os.path.basename(d) for d in B._includes(os.path.join(B.CSRC, "plan.cpp"))}
    assert "pencil_b200.h" in deps and "pb_internal.hpp" in deps


def test_stale_follows_the_newest_dependency(tmp_path):
    target = tmp_path / "a.o"
    dep = tmp_path / "a.hpp"
    dep.write_text("x")
    target.write_text("o")
    os.utime(dep, (1000, 1000))
    os.utime(target, (2000, 2000))
    assert not B._stale(str(target), [str(dep)])
    os.utime(dep, (3000, 3000))
    assert B._stale(str(target), [str(dep)])
    assert B._stale(str(tmp_path / "missing.o"), [str(dep)])
