"""Build the CUDA library (liblsb.so) in-tree for sm_100a.

The library is plain nvcc output: every .cu under csrc/ compiled for
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared object
that exports the C-ABI of include/lsb.h.  No JIT cache, no torch extension:
the .so sits next to this file so it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblsb.so"
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build liblsb.so")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile liblsb.so if it is missing or older than its sources."""
    if not force and not needs_build():
        return LIB
    cmd = [
        nvcc_path(), "-std=c++17", "-O3", "-lineinfo", *ARCH_FLAGS,
        "-I", str(ROOT / "include"), "-Xcompiler", "-fPIC", "-shared",
        "-o", str(LIB) + ".tmp", *map(str, sources()),
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
