"""Build the native libraries in-tree.

* ``glp_b200/libglp_b200.so`` -- the CUDA engine (sm_100a) behind the C ABI of
  ``include/glp.h``;
* ``oracle/liboracle.so`` -- the CPU oracle (test infrastructure only);
* ``glp_b200/glp_cli`` -- the command line driver mirroring the reference's
  ``GPULP method niter in out ifdirect`` (main.cu:38-56).

Run ``python -m glp_b200.build`` (or ``__graft_entry__.build()``).  nvcc
cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "glp_b200")
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libglp_b200.so")
CLI = os.path.join(PKG, "glp_cli")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp"]
ENGINE_SOURCES = ["engine.cu", "graphgen.cu", "batch.cu", "server.cu", "ingest.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _deps(directory: str, exts=(".cu", ".cuh", ".h", ".cpp")) -> list[str]:
    out = []
    for d in (directory, os.path.join(ROOT, "include")):
        for f in sorted(os.listdir(d)):
            if f.endswith(exts):
                out.append(os.path.join(d, f))
    return out


def build_engine(force: bool = False, verbose_ptxas: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in ENGINE_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if not force and _newer(LIB, _deps(CSRC)):
        return LIB
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    _run([_nvcc(), *NVCC_ARCH, *NVCC_FLAGS, *extra, "-shared", *srcs, "-o", LIB, "-lgomp"])
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "cli.cpp")
    if not os.path.exists(src):
        return ""
    if not force and _newer(CLI, [src, LIB, os.path.join(ROOT, "include", "glp.h")]):
        return CLI
    _run(["g++", "-O2", "-std=c++17", src, "-o", CLI, f"-I{ROOT}/include", f"-L{PKG}", "-lglp_b200",
          "-Wl,-rpath,$ORIGIN"])
    return CLI


def build_oracle(force: bool = False) -> str:
    src = os.path.join(ROOT, "oracle", "glp_oracle.cpp")
    if not force and _newer(ORACLE_LIB, [src]):
        return ORACLE_LIB
    _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", src, "-o", ORACLE_LIB])
    return ORACLE_LIB


def build_all(force: bool = False) -> None:
    build_engine(force)
    build_cli(force)
    build_oracle(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
