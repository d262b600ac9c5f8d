"""Build the product library libses_b200.so (sm_100a) in-tree with nvcc.

Usage: ``python shoeridingerequationsolver_b200/build.py [--verbose-ptxas]`` (runs
without importing the package, which needs the built library).
The library exports exactly the C ABI declared in ``include/ses_gpu.h``.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libses_b200.so"
SOURCES = ["ses_gpu.cu", "ses_plans_small.cu", "ses_plans_mixed.cu", "ses_plans_256.cu",
           "ses_plans_large.cu", "ses_plans_plane.cu", "ses_noalloc.cu", "ses_serve.cpp"]
HEADERS = ["ses_fft.cuh", "ses_pass.cuh", "ses_pass2.cuh", "ses_pass3.cuh", "ses_tma.cuh", "ses_plans.cuh", "ses_engine.cuh",
           "ses_aux.cuh", "ses_plane.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-shared",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fvisibility=hidden"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "ses_gpu.h"]
    return all(d.stat().st_mtime <= t for d in deps)


def includes(path: Path, seen=None) -> set:
    """The quoted #include files of a source, followed recursively inside csrc/ and include/."""
    seen = set() if seen is None else seen
    for line in path.read_text().splitlines():
        line = line.strip()
        if not line.startswith('#include "'):
            continue
        name = line.split('"')[1]
        for d in (CSRC, ROOT / "include"):
            f = d / name
            if f.exists() and f not in seen:
                seen.add(f)
                includes(f, seen)
    return seen


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile each out-of-date translation unit in parallel, then link the shared library."""
    if not force and up_to_date():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    compile_flags = [f for f in FLAGS if f != "-shared"]
    procs, objs = [], []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        objs.append(obj)
        deps = [CSRC / src, Path(__file__), *includes(CSRC / src)]
        if not force and obj.exists() and all(d.stat().st_mtime <= obj.stat().st_mtime for d in deps):
            continue
        cmd = [nvcc(), *ARCH, *compile_flags, "-I", str(ROOT / "include"), "-I", str(CSRC), "-c",
               str(CSRC / src), "-o", str(obj)]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((obj, subprocess.Popen(cmd)))
    failed = [str(o) for o, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    link = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *[str(o) for o in objs], "-o", str(LIB)]
    subprocess.run(link, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force or args.verbose_ptxas, ptxas_verbose=args.verbose_ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
