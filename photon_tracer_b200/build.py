"""Builds libphoton_cuda.so in-tree: CUDA sources with nvcc for sm_100a, host
C++ with g++, linked into one shared library beside this file.

Float code is compiled without contraction on both sides (-fmad=false for the
device, -ffp-contract=off for the host) and with IEEE division and square
root, because closest hits must match the reference bit for bit.

    python -m photon_tracer_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libphoton_cuda.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I" + os.path.join(ROOT, "include"),
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-Wno-unused-parameter",
             "-I" + os.path.join(CUDA_HOME, "include"), "-I" + os.path.join(ROOT, "include")]


def _sources():
    cu, cpp = [], []
    for name in sorted(os.listdir(CSRC)):
        path = os.path.join(CSRC, name)
        if name.endswith(".cu"):
            cu.append(path)
        elif name.endswith(".cpp"):
            cpp.append(path)
    return cu, cpp


def _headers():
    out = [os.path.join(ROOT, "include", "photon_cuda.h")]
    for name in os.listdir(CSRC):
        if name.endswith((".h", ".hpp", ".cuh")):
            out.append(os.path.join(CSRC, name))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed ({res.returncode}): {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose and (res.stdout or res.stderr):
        print(res.stdout, res.stderr, flush=True)
    return res


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False, defines=(), out_dir=None) -> str:
    """Compiles what changed and links the library; returns its path.
    defines (e.g. ["PT_MEGA_MIN_BLOCKS=5"]) and out_dir build a tuning
    variant elsewhere instead of the in-tree library."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    build_dir = os.path.join(out_dir, "_build") if out_dir else BUILD
    lib_path = os.path.join(out_dir, "libphoton_cuda.so") if out_dir else LIB
    dflags = ["-D" + d for d in defines]
    os.makedirs(build_dir, exist_ok=True)
    cu, cpp = _sources()
    headers = _headers()
    jobs, objs = [], []
    for src in cu:
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            jobs.append([NVCC] + NVCC_FLAGS + dflags + extra + ["-c", src, "-o", obj])
    for src in cpp:
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append(["g++"] + CXX_FLAGS + dflags + ["-c", src, "-o", obj])
    outputs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            outputs = list(ex.map(lambda c: _run(c, verbose), jobs))
    if ptxas_verbose:
        for r in outputs:
            sys.stdout.write(r.stderr)
    if force or jobs or _stale(lib_path, objs):
        tmp = lib_path + ".tmp"
        _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"],
             verbose)
        shutil.move(tmp, lib_path)
    return lib_path


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill reports")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose, ptxas_verbose=args.ptxas))


if __name__ == "__main__":
    main()
