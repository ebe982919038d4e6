"""Builds the engine's shared library in-tree (sm_100a) and, for the tests,
the host oracle.

    python -m cudacode_b200.build            # engine + oracle
    python -m cudacode_b200.build --engine   # engine only

The engine library ``cudacode_b200/libpyro.so`` is built with nvcc for
``sm_100a`` only; the update kernels are compiled with ``--fmad=false`` so
that every fused multiply-add is the explicit ``fmaf`` of
``include/pyro_math.h`` and they round exactly like the host oracle (the
learned move's kernels, checked against the oracle by tolerance, are not).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpyro.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")

ENGINE_SOURCES = ["kernels.cu", "j1_kernels.cu", "far_kernels.cu", "gen_wave.cu", "sq_kernels.cu", "tet_mlp.cu", "smem_kernels.cu",
                  "capi.cu",
                  "tet_capi.cu", "checkpoint.cu", "lattice.cpp", "noalloc.cu", "exchange.cu", "order.cu", "tet_umma.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FMAD_SOURCES = {"tet_mlp.cu", "tet_umma.cu"}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the engine needs the CUDA 12.9 toolkit")
    return cand


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _deps() -> list[str]:
    out = [os.path.abspath(__file__)]  # flag changes rebuild too
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".cpp", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def build_engine(force: bool = False, verbose: bool = False) -> str:
    deps = _deps()
    if not force and _newer(LIB, deps):
        return LIB
    objs = []
    build_dir = os.path.join(PKG, "_build")
    os.makedirs(build_dir, exist_ok=True)
    common = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I", os.path.join(ROOT, "include")]
    cmds = []
    for src in ENGINE_SOURCES:
        obj = os.path.join(build_dir, src.rsplit(".", 1)[0] + ".o")
        # The learned move's kernels agree with the oracle by tolerance (BF16
        # network, FP32 proposals), so they may contract multiply-adds; every
        # other kernel is bit-exact with the oracle and keeps --fmad=false.
        fmad = [] if src in FMAD_SOURCES else ["--fmad=false"]
        cmd = [*common, *fmad, "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [*common, *fmad, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # Translation units compile independently: one nvcc per source, in parallel.
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for res in pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise subprocess.CalledProcessError(res.returncode, res.args)
            if verbose and (res.stdout or res.stderr):
                sys.stderr.write(res.stdout + res.stderr)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


CLI = os.path.join(PKG, "pyro_run")


def build_cli(force: bool = False) -> str:
    """The C++ command-line driver (host code only), linked to libpyro.so."""
    src = os.path.join(PKG, "host", "pyro_run.cpp")
    deps = [src, os.path.join(PKG, "host", "pyro_host.hpp"), os.path.join(PKG, "host", "measure.hpp"),
            os.path.join(ROOT, "include", "pyro.h"), LIB]
    if not force and _newer(CLI, deps):
        return CLI
    cxx = shutil.which("g++") or "/usr/bin/g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", src, "-o", CLI, "-L", PKG, "-lpyro",
                    "-Wl,-rpath,$ORIGIN", "-Wl,--enable-new-dtags"], check=True)
    return CLI


def build_oracle(force: bool = False) -> str:
    """Compiles the host oracle (test infrastructure) with make."""
    subprocess.run(["make", "-s", "-C", ORACLE_DIR] + (["-B"] if force else []), check=True)
    return os.path.join(ORACLE_DIR, "liboracle.so")


def main(argv: list[str]) -> int:
    force = "--force" in argv
    build_engine(force=force, verbose="-v" in argv)
    build_cli(force=force)
    if "--engine" not in argv:
        build_oracle(force=force)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
