"""Compile libdgann.so (the sm_100a search library) in-tree.

Usage: python -m pydiskann_b200.build [--force] [-j N]

Every translation unit under csrc/ is compiled by nvcc for sm_100a in
parallel and linked into pydiskann_b200/libdgann.so, next to this file, so
the library travels with the source tree.  The index-construction units
(medoid, Vamana build, PQ training and encodes, exact kNN) are also linked on
their own into libdgbuild.so, which a process that only prepares an index
loads instead of the search library.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdgann.so")
BUILD_LIB = os.path.join(HERE, "libdgbuild.so")
BUILD_UNITS = ("dg_errors", "dg_build", "dg_vamana")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", INCLUDE] + ARCH


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "dgann.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False, defines=(),
          obj_dir: str | None = None, lib_path: str | None = None) -> str:
    """Compile every csrc/*.cu and link the library (only stale objects rebuild).

    `defines` adds -D flags (tuning knobs such as DG_SEARCH_MIN_BLOCKS);
    obj_dir / lib_path place an alternative build elsewhere.
    """
    OBJ_ = obj_dir or OBJ
    LIB_ = lib_path or LIB
    os.makedirs(OBJ_, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    srcs = _sources()
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(OBJ_, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        cmd = [nvcc] + NVCC_FLAGS + [f"-D{d}" for d in defines] + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {s}:\n{r.stderr[-6000:]}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return o

    if todo:
        jobs = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(jobs) as ex:
            list(ex.map(compile_one, todo))
    links = [(LIB_, objs)]
    if lib_path is None:
        links.append((BUILD_LIB, [o for o in objs if os.path.basename(o)[:-2] in BUILD_UNITS]))
    for target, parts in links:
        if force or todo or _stale(target, parts):
            cmd = [nvcc] + ARCH + ["-shared", "-o", target] + parts + ["-lcudart", "-Xlinker", "--no-undefined"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link of {os.path.basename(target)} failed:\n{r.stderr[-4000:]}")
    return LIB_


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    ap.add_argument("-D", action="append", default=[], help="extra preprocessor define")
    ap.add_argument("--obj-dir", default=None)
    ap.add_argument("--lib", default=None)
    a = ap.parse_args()
    print(build(a.force, a.j, a.v, a.D, a.obj_dir, a.lib))
