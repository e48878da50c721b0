"""Build the B200 back end in-tree: pcbroute_b200/lib/libpcbgpu.so (sm_100a) and the CPU oracle library.

    python -m pcbroute_b200.build            # both
    python -m pcbroute_b200.build --no-oracle

nvcc compiles every kernel for sm_100a only (-gencode arch=compute_100a,code=sm_100a); there is no other target
and no fallback. Floating-point contraction is off everywhere: the fixed-point weights are defined by single IEEE
multiplies, and the oracle (built with -ffp-contract=off) must agree bit for bit.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pcbroute_b200")
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libpcbgpu.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "libpcboracle.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["solver.cu", "query.cu", "batcher.cpp", "synth.cu", "costs.cu", "spec.cu", "mlp.cu", "sched.cu", "mirror.cu",
           "gpu_api.cpp"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_lib(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, "pcbg_internal.h"), os.path.join(ROOT, "include", "pcbg.h"),
                   os.path.join(ROOT, "include", "gpu.h"), __file__]
    if not force and _newer(LIB, deps):
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [NVCC, *ARCH, *common, "-c", s, "-o", o]
        if verbose_ptxas and s.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        _run(cmd)
        objs.append(o)
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


def build_oracle(force: bool = False) -> str:
    src = os.path.join(ORACLE_DIR, "pcb_oracle.c")
    deps = [src, os.path.join(ORACLE_DIR, "pcb_oracle.h"), os.path.join(ROOT, "include", "pcbg.h")]
    if not force and _newer(ORACLE_LIB, deps):
        return ORACLE_LIB
    os.makedirs(os.path.dirname(ORACLE_LIB), exist_ok=True)
    tmp = ORACLE_LIB + ".tmp"
    _run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-o", tmp, src, "-lm", "-lpthread"])
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build_lib(a.force, a.ptxas_v))
    if not a.no_oracle:
        print(build_oracle(a.force))


if __name__ == "__main__":
    main()
