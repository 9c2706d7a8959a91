"""Builds libcg_cuda.so in-tree for sm_100a.

    python -m crystalgraphics_b200.build        (or build() from Python)

Every .cu/.cpp under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; host code gets
``-ffp-contract=off`` (the host packing must round exactly like the code it
restates).  Objects go to crystalgraphics_b200/_build/, the library to
crystalgraphics_b200/libcg_cuda.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
# CG_NVCC_DEFINES (e.g. "CG_SMITS_SHARED" or "CG_STEP_BUDGET=8"): preprocessor
# switches of a kernel variant for measurements; such builds keep their objects
# apart
DEFINES = os.environ.get("CG_NVCC_DEFINES", "").split()
BUILD = os.path.join(HERE, "_build" + ("_" + "_".join(DEFINES).replace("=", "-") if DEFINES else ""))
LIB = os.path.join(HERE, "libcg_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags(extra_device: list[str] | None = None) -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++20", "--expt-relaxed-constexpr",
                   "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
                   "-I", os.path.join(HERE, "..", "include")] + ["-D" + d for d in DEFINES] + \
        (extra_device or [])


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str, verbose: bool, ptxas_v: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "cg_cuda.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps) \
            and not ptxas_v:
        return obj
    cmd = [nvcc(), "-c", src, "-o", obj] + _flags(["-Xptxas", "-v"] if ptxas_v else None)
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "cu", "-c", src, "-o", obj] + _flags()
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if ptxas_v and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


CXX_DIR = os.path.join(HERE, "cxx")
CXX_LIB = os.path.join(HERE, "libcrystalgraphics.so")
CXX_EXE = os.path.join(HERE, "cg_view")


def _stale(out: str, deps: list[str]) -> bool:
    return not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps)


def build_cxx(verbose: bool = False) -> str:
    """The C++23 crystal::graphics layer (libcrystalgraphics.so) and the
    headless example program (cg_view), linked against libcg_cuda.so."""
    inc = os.path.join(HERE, "..", "include")
    headers = [os.path.join(inc, "cg_cuda.h")] + [
        os.path.join(inc, "CrystalGraphics", f) for f in os.listdir(os.path.join(inc, "CrystalGraphics"))]
    cxx = os.environ.get("CXX", "g++")
    common = ["-std=c++23", "-O2", "-fPIC", "-I", inc, "-I", os.path.join(inc, "CrystalGraphics", "..")]
    src = os.path.join(CXX_DIR, "crystal_graphics.cpp")
    if _stale(CXX_LIB, [src, LIB] + headers):
        cmd = [cxx] + common + ["-shared", "-o", CXX_LIB, src, "-L", HERE, "-l:libcg_cuda.so",
                                "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    main = os.path.join(CXX_DIR, "view_main.cpp")
    if _stale(CXX_EXE, [main, CXX_LIB] + headers):
        cmd = [cxx] + common + ["-o", CXX_EXE, main, "-L", HERE, "-l:libcrystalgraphics.so",
                                "-l:libcg_cuda.so", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return CXX_LIB


def build(verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, ptxas_v), srcs))
    stamp = LIB + ".variant"  # the switches the library was linked with
    variant = " ".join(DEFINES)
    same = os.path.exists(stamp) and open(stamp).read() == variant
    if not same or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB)
                                                  for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-lcudart", "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
        with open(stamp, "w") as f:
            f.write(variant)
    build_cxx(verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_v="-v" in sys.argv))
