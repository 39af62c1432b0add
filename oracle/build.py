"""TEST INFRASTRUCTURE: builds the checkers the tests use.

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


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build_oracle(args.force))
    print(build_ref(args.force) or "reference checkout absent: oracle/_ref not built")


if __name__ == "__main__":
    sys.exit(main())
