"""TEST INFRASTRUCTURE: builds the libraries the tests compare against.

* oracle/libptoracle.so -- the plain-C restatement (pt_oracle.c), always.
* oracle/_ref/libptref.so -- the reference itself: ref_harness.cpp compiled
  against the reference's own headers where they lie (PT_REFERENCE_DIR,
  default /root/reference), with the reference's Makefile flags
  (-O3 -std=c++17 -pthread, no -march) plus -ffp-contract=off. Skipped when
  the reference checkout is absent (the prebuilt .so is used if present).

Nothing here is shipped: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg load these libraries.

    python oracle/build.py [--force]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ORACLE_LIB = os.path.join(HERE, "libptoracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libptref.so")
REFERENCE = os.environ.get("PT_REFERENCE_DIR", "/root/reference")


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(d) > os.path.getmtime(target) for d in deps)


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build_oracle(force=False):
    src = os.path.join(HERE, "pt_oracle.c")
    hdr = os.path.join(ROOT, "include", "photon_cuda.h")
    if force or _stale(ORACLE_LIB, [src, hdr, __file__]):
        _run(["gcc", "-O2", "-std=c99", "-D_DEFAULT_SOURCE", "-fPIC", "-shared", "-ffp-contract=off", "-Wall",
              "-o", ORACLE_LIB, src, "-lm"])
    return ORACLE_LIB


def build_ref(force=False):
    """Builds oracle/_ref/libptref.so when the reference checkout is present."""
    inc = os.path.join(REFERENCE, "include")
    if not os.path.isdir(inc):
        return REF_LIB if os.path.exists(REF_LIB) else None
    src = os.path.join(HERE, "ref_harness.cpp")
    deps = [src, os.path.join(ROOT, "include", "photon_cuda.h"), __file__]
    deps += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".hpp")]
    os.makedirs(REF_DIR, exist_ok=True)
    if force or _stale(REF_LIB, deps):
        _run(["g++", "-std=c++17", "-O3", "-pthread", "-ffp-contract=off", "-fPIC", "-shared", "-w",
              "-I" + inc, "-o", REF_LIB, src])
    return REF_LIB


def build_shim_check(force=False):
    """oracle/_ref/shim_check: include/photon_cuda_geometry.hpp driven by the
    reference's own scenes, linked against the product library."""
    inc = os.path.join(REFERENCE, "include")
    out = os.path.join(REF_DIR, "shim_check")
    lib_dir = os.path.join(ROOT, "photon_tracer_b200")
    if not os.path.isdir(inc) or not os.path.exists(os.path.join(lib_dir, "libphoton_cuda.so")):
        return out if os.path.exists(out) else None
    src = os.path.join(HERE, "shim_check.cpp")
    deps = [src, os.path.join(ROOT, "include", "photon_cuda.h"), os.path.join(ROOT, "include", "photon_cuda_geometry.hpp"),
            os.path.join(lib_dir, "libphoton_cuda.so"), __file__]
    os.makedirs(REF_DIR, exist_ok=True)
    if force or _stale(out, deps):
        _run(["g++", "-std=c++17", "-O2", "-pthread", "-ffp-contract=off", "-w", "-I" + inc, "-o", out, src,
              "-L" + lib_dir, "-lphoton_cuda", "-Wl,-rpath,$ORIGIN/../../photon_tracer_b200"])
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build_oracle(args.force))
    print(build_ref(args.force) or "reference checkout absent: oracle/_ref not built")
    print(build_shim_check(args.force) or "shim check not built")


if __name__ == "__main__":
    sys.exit(main())
