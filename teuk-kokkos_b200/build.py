"""Build the B200 engine shared library in-tree.

    python teuk-kokkos_b200/build.py [--force] [--verbose]

Compiles csrc/*.cu and csrc/*.cpp with nvcc for sm_100a only into
teuk-kokkos_b200/lib/libteuk_b200.so (CUDA runtime linked statically, so the
library needs only the driver at run time).  The build cross-compiles without
a GPU.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIB_DIR = PACKAGE / "lib"
LIBRARY = LIB_DIR / "libteuk_b200.so"
SOURCES = ["plan.cpp", "checkpoint.cpp", "run_config.cpp", "kernels.cu",
           "second_order.cu",
           "static_scratch.cu", "api.cu"]
HEADERS = ["engine.h", "kernels.h", "second_order.h", "stream_kernel.cuh", "static_scratch.h",
           "checkpoint.h", "run_config.h", "sbp_tables.h", "split_precision.cuh"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    found = shutil.which("nvcc")
    if found:
        return found
    candidate = Path("/usr/local/cuda/bin/nvcc")
    if candidate.exists():
        return str(candidate)
    raise RuntimeError("nvcc not found: the B200 engine cannot be built")


def _stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = [CSRC / s for s in SOURCES + HEADERS] + [REPO / "include" / "teuk_b200.h",
                                                      Path(__file__)]
    return any(p.stat().st_mtime > built for p in inputs)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> Path:
    if not force and not _stale():
        return LIBRARY
    LIB_DIR.mkdir(exist_ok=True)
    cmd = [nvcc_path(), *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++20",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-shared",
           "--expt-relaxed-constexpr",
           "-I", str(REPO / "include"), "-I", str(CSRC),
           "-o", str(LIBRARY) + ".tmp",
           *[str(CSRC / s) for s in SOURCES]]
    if extra_flags:
        cmd[1:1] = list(extra_flags)
    if verbose:
        print(" ".join(cmd), flush=True)
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError("nvcc failed building libteuk_b200.so")
    if verbose and (result.stdout or result.stderr):
        print(result.stdout + result.stderr)
    os.replace(str(LIBRARY) + ".tmp", LIBRARY)
    return LIBRARY


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true")
    parser.add_argument("--ptxas-verbose", action="store_true",
                        help="print register / shared-memory use per kernel")
    args = parser.parse_args()
    extra = ["-Xptxas", "-v"] if args.ptxas_verbose else None
    path = build(force=args.force or args.ptxas_verbose, verbose=args.verbose or
                 args.ptxas_verbose, extra_flags=extra)
    print(path)


if __name__ == "__main__":
    main()
