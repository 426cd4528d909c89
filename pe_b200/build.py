"""Builds libpe_b200.so in-tree (pe_b200/libpe_b200.so) from pe_b200/csrc/*.cu for sm_100a.

Usage: python -m pe_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpe_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-fopenmp", "--expt-relaxed-constexpr",
              "-I" + INCLUDE]
# per-file flags: the box fine detection rounds every product and sum separately, as pe's FP64
# code does (its case selection compares depths that tie for aligned boxes); so do the
# hard-contact kernels and the DEM step and list rebuild kernels, whose forms must give the same
# bits in every kernel they are compiled into (contracted multiply-adds are chosen per kernel by
# the compiler, and a kernel's launch bounds changed its choices)
FILE_FLAGS = {"boxes.cu": ["-fmad=false"], "nbgs.cu": ["-fmad=false"], "dem.cu": ["-fmad=false"],
              "rebuild.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "pe_b200.h"))
    return hs


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    return os.path.getmtime(LIB) >= _newest(sources() + headers() + [__file__])


def build(force: bool = False, verbose: bool = False, extra_flags=(), out: str = None,
          build_dir: str = None) -> str:
    lib = out or LIB
    bdir = build_dir or BUILD
    if out is None and not force and up_to_date():
        return LIB
    os.makedirs(bdir, exist_ok=True)
    cc = nvcc()
    objs = []

    def compile_one(src):
        obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
        cmd = [cc, *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(os.path.basename(src), []), *extra_flags,
               "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = lib + ".tmp"
    cmd = [cc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-Xcompiler", "-fopenmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=force or bool(extra), verbose=verbose or bool(extra), extra_flags=extra))
