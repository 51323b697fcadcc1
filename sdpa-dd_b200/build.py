"""Build the sm_100a library and the command-line driver in-tree.

    python sdpa-dd_b200/build.py [-j N] [--force]

Outputs (git-ignored, shipped with the tree):
    sdpa-dd_b200/lib/libsddd.so      C ABI of include/sddd.h
    sdpa-dd_b200/bin/sdpa_dd_b200    drop-in for the reference's sdpa_dd
Objects go to sdpa-dd_b200/_build/.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
SRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libsddd.so"
BIN = PKG / "bin" / "sdpa_dd_b200"

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
HOSTCXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# dd arithmetic must round exactly as written: no contraction anywhere
FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-ccbin", HOSTCXX,
                "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I", str(PKG.parent / "include")]
LIB_SOURCES = ["prof.cu", "blas.cu", "schur.cu", "newton.cu", "eig.cu", "context.cu", "ddkern.cu", "noalloc.cu", "ozaki.cu", "ozaki_gemm.cu", "batched.cu", "trsv_blocked.cu", "adjoint.cu", "sparse_chol.cu", "sparse_schur.cpp",
               "problem.cpp", "solver.cpp", "capi.cpp", "cli.cpp", "batch.cpp"]


def _compile(src: pathlib.Path, obj: pathlib.Path, force: bool) -> str:
    deps = [src] + sorted(SRC.glob("*.h")) + sorted(SRC.glob("*.cuh")) + [PKG.parent / "include" / "sddd.h"]
    if not force and obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return ""
    cmd = [NVCC] + FLAGS + ["-x", "cu", "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr}")
    return src.name


def build(jobs: int = 8, force: bool = False, verbose: bool = True) -> None:
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    BIN.parent.mkdir(exist_ok=True)
    objs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = []
        for name in LIB_SOURCES + ["main.cpp"]:
            src = SRC / name
            obj = OBJ / (name.rsplit(".", 1)[0] + ".o")
            futs.append(ex.submit(_compile, src, obj, force))
            if name != "main.cpp":
                objs.append(obj)
        for f in futs:
            done = f.result()
            if done and verbose:
                print(f"  compiled {done}", file=sys.stderr)
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        subprocess.run([NVCC] + ARCH + ["-shared", "-ccbin", HOSTCXX, "-o", str(LIB)] + [str(o) for o in objs],
                       check=True)
    main_o = OBJ / "main.o"
    if force or not BIN.exists() or BIN.stat().st_mtime < max(LIB.stat().st_mtime, main_o.stat().st_mtime):
        subprocess.run([NVCC] + ARCH + ["-ccbin", HOSTCXX, "-o", str(BIN), str(main_o), "-L", str(LIB.parent), "-lsddd",
                        "-Xlinker", "-rpath,$ORIGIN/../lib"], check=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(a.j, a.force)
    print(LIB)
    print(BIN)
