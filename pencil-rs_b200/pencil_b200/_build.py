"""Build the sm_100a shared library ``libpencil_b200.so`` in-tree with nvcc.

``python -m pencil_b200._build`` (from ``pencil-rs_b200/``) or
``__graft_entry__.build()``.  Objects go to ``pencil-rs_b200/_build/``; the
library is written next to this file so it travels with the source tree.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(ROOT), "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libpencil_b200.so")

# (source, object, preprocessor definitions): mr_kernels.cu is compiled once
# per group of lengths (MR_GROUPS in mr_lengths.hpp) and mr_bs_kernels.cu once
# per kernel kind and layout variant, so the groups build in parallel
MR_GROUPS = 8
# the longest compilations first, so that a full build keeps every core busy
# to the end
SOURCES = ([("pass_kernel.cu", "pass_kernel.cu.o", [])]
           + [("mr_kernels.cu", f"mr_kernels_g{g}.o", [f"-DMR_GROUP={g}"]) for g in range(MR_GROUPS)]
           + [("mr_r2r_kernels.cu", f"mr_r2r_kernels_g{g}.o", [f"-DMR_GROUP={g}"]) for g in range(MR_GROUPS)]
           + [("mr_bs_kernels.cu", f"mr_bs_kernels_k{k}v{v}.o", [f"-DBS_KIND={k}", f"-DBS_V={v}"])
              for k in (1, 2) for v in (0, 1, 2)]
           + [(s, s + ".o", []) for s in ("pow2_kernel.cu", "plan.cpp", "field_ops.cu", "aux_kernels.cu",
                                         "no_alloc.cu", "mr_dispatch.cpp")])
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _includes(path: str, seen=None) -> set:
    """The project headers a source includes, directly or through other
    headers (quoted includes found in csrc/ or include/)."""
    seen = set() if seen is None else seen
    with open(path) as f:
        text = f.read()
    for name in _INCLUDE_RE.findall(text):
        for d in (os.path.dirname(path), CSRC, INCLUDE):
            cand = os.path.join(d, name)
            if os.path.exists(cand):
                cand = os.path.abspath(cand)
                if cand not in seen:
                    seen.add(cand)
                    _includes(cand, seen)
                break
    return seen


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs, cmds = [], []
    for src, oname, defs in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, oname)
        objs.append(obj)
        if force or _stale(obj, [path, *sorted(_includes(path))]):
            cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
                   "-I", CSRC, *defs, "-c", path, "-o", obj]
            if src.endswith(".cu"):
                cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
            if verbose:
                print(" ".join(cmd), flush=True)
            cmds.append(cmd)
    jobs = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as pool:
        for proc in list(pool.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), cmds)):
            if proc.returncode != 0:
                sys.stderr.write(proc.stderr or "")
                raise subprocess.CalledProcessError(proc.returncode, proc.args)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
