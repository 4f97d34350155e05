"""The source-compatible C++ header (include/lslab_compat.h): a caller in the
reference's style compiles and links against liblsb.so on the CPU; the GPU
test runs it."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "compat" / "compat_smoke.cpp"
CUDA = Path("/usr/local/cuda")


def _build(tmp: Path) -> Path:
    exe = tmp / "compat_smoke"
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-I", str(CUDA / "include"),
           str(SRC), "-o", str(exe), "-L", str(ROOT / "lslab_b200"), "-llsb",
           "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{ROOT / 'lslab_b200'}",
           f"-Wl,-rpath,{CUDA / 'lib64'}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_compat_header_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_compat_header_runs(tmp_path, cuda):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "compat ok" in r.stdout
