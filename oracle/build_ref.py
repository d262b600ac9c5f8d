"""Build recipe: compile the reference's own FP64 CPU core into oracle/_ref/libsesref.so.

This is test infrastructure. It reads the reference sources where they lie
(``$SES_REF``, default ``/root/reference``), rewrites their C++20 named-module
lines into plain header lines (g++ 13 cannot build the modules), and writes the
result only under ``oracle/_ref/`` (git-ignored).  Nothing from the reference
is committed.

The rewrite is mechanical and touches no statement of the algorithm:

* ``module;`` global-fragment marker           -> dropped
* ``export module ses.<m>;``                   -> ``#pragma once``
* ``[export ] import ses.<m>;``                -> ``#include "<m>.hpp"``
* ``export namespace``                         -> ``namespace``
* ``Pool& pool() {`` (parallel.ixx:172)         -> ``inline Pool& pool() {``
  (a module-linkage function becomes an inline header function; one pool per
  process either way)

The shimmed headers are compiled together with ``oracle/ref_capi.cpp`` (a C
wrapper written for this repository around the reference's public C++ API)
using the reference's own numeric flags (reference CMakeLists.txt:59-112):
``-O2 -mavx2 -mfma -ffp-contract=off -fcx-limited-range``.

Usage: ``python oracle/build_ref.py [--ref DIR]``.  Exits 0 and prints
``skipped`` when the reference tree is absent (the GPU box only uses the
prebuilt library that travels with the repository snapshot).
"""

from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
GEN = OUT / "gen"
LIB = OUT / "libsesref.so"

# Reference core modules on the split-operator path (core/src/<m>.ixx).
MODULES = [
    "grid", "vec", "parallel", "field", "spectral", "fft", "propagator",
    "potential", "wavepacket", "observables", "imaginary_time", "drive",
]

FLAGS = ["-std=c++20", "-O2", "-mavx2", "-mfma", "-ffp-contract=off",
         "-fcx-limited-range", "-fPIC", "-shared", "-pthread"]

_IMPORT = re.compile(r"^\s*(?:export\s+)?import\s+ses\.([a-z_0-9]+)\s*;\s*$")
_MODULE = re.compile(r"^\s*export\s+module\s+ses\.[a-z_0-9]+\s*;\s*$")


def shim_module(text: str) -> str:
    out = []
    for line in text.splitlines():
        if line.strip() == "module;":
            continue
        if _MODULE.match(line):
            out.append("#pragma once")
            continue
        m = _IMPORT.match(line)
        if m:
            out.append(f'#include "{m.group(1)}.hpp"')
            continue
        line = re.sub(r"^(\s*)export\s+namespace\b", r"\1namespace", line)
        if re.match(r"^Pool&\s+pool\(\)\s*\{", line):
            line = "inline " + line
        out.append(line)
    return "\n".join(out) + "\n"


def generate(ref: Path) -> None:
    GEN.mkdir(parents=True, exist_ok=True)
    for m in MODULES:
        src = ref / "core" / "src" / f"{m}.ixx"
        (GEN / f"{m}.hpp").write_text(shim_module(src.read_text()))


def build(ref: Path, cxx: str = "g++") -> Path:
    generate(ref)
    cmd = [cxx, *FLAGS, "-I", str(GEN), str(HERE / "ref_capi.cpp"), "-o", str(LIB)]
    subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SES_REF", "/root/reference"))
    args = ap.parse_args(argv)
    ref = Path(args.ref)
    if not (ref / "core" / "src" / "propagator.ixx").exists():
        print(f"skipped: reference tree not found at {ref}")
        return 0
    lib = build(ref)
    print(f"built {lib}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
