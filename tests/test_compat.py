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


def _reference_benchmark() -> Path | None:
    import oracle
    inc = oracle.reference_include()
    if inc is None:
        return None
    src = inc.parent / "benchmark" / "benchmark.cu"
    return src if src.exists() else None


def test_reference_benchmark_compiles_unchanged(tmp_path):
    """The reference's own caller, benchmark/benchmark.cu (its
    lslab::map<unsigned long long, unsigned>, thrust buffers, gpuErrchk),
    compiled as it is against include/compat (<lslab/map.h> resolves to this
    library's front) and linked with liblsb.so."""
    src = _reference_benchmark()
    if src is None:
        pytest.skip("reference sources not present (set LSLAB_REFERENCE)")
    exe = tmp_path / "benchmark_on_lsb"
    nvcc = shutil.which("nvcc") or str(CUDA / "bin" / "nvcc")
    cmd = [nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include" / "compat"), "-I", str(ROOT / "include"), str(src),
           "-o", str(exe), "-L", str(ROOT / "lslab_b200"), "-llsb"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert exe.exists()


@pytest.mark.gpu
def test_reference_benchmark_runs_on_lsb(cuda):
    """The reference's benchmark built unchanged against this library
    (oracle/_ref/benchmark_on_lsb, made by `make -C oracle ref`) runs its
    populate, 10 get batches and 10 put batches to completion."""
    exe = ROOT / "oracle" / "_ref" / "benchmark_on_lsb"
    assert exe.exists(), "oracle/_ref/benchmark_on_lsb is missing (make -C oracle ref)"
    r = subprocess.run([str(exe), "-s", "16", "-p", "30000", "-b", "4096", "-r", "60000",
                        "-c", "256"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert r.stdout.count("Throughput") == 20, r.stdout[-2000:]
    assert "---- Get -----" in r.stdout and "---- Put -----" in r.stdout
