"""Build the CUDA library libahop_b200.so in-tree for sm_100a (B200).

Every translation unit is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into
one shared library next to this file, so the built artefact travels with the
source tree.  The finder's ranking arithmetic (distances, densities, saddle
and threshold tests) is written with explicitly rounded intrinsics, and the
finder files are also compiled with -fmad=false so that no other expression
in them is contracted into a fused multiply-add.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
REPO = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(HERE, "libahop_b200.so")

FINDER_SOURCES = ["knn.cu", "hop.cu", "saddle.cu", "forest.cu", "nodes.cu", "msm.cu", "adjoint.cu", "capi.cu"]
PROPS_SOURCES = ["halo_props.cu", "halo_virial.cu", "ramses.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return [s for s in FINDER_SOURCES + PROPS_SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    common = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
    jobs = []
    for src in _sources():
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        path = os.path.join(CSRC, src)
        if force or _stale(obj, path):
            flags = ["-fmad=false"] if src in FINDER_SOURCES else []
            jobs.append(common + flags + ["-c", path, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    objs = [os.path.join(BUILD, s.replace(".cu", ".o")) for s in _sources()]
    if force or jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lcuda"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
