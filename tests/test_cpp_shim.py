"""The C++ PhotonMap / KDTreePoint shim (include/pmgpu.hpp): it compiles
against the C ABI (CPU), and on a GPU the reference-shaped call sequence gives
the same bits as direct C-ABI calls (tests/cpp/shim_test.cpp)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "shim_test.cpp"


def nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def test_shim_header_compiles():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(ROOT / "include"), "-I",
                        "/usr/local/cuda/include", str(SRC)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_shim_matches_c_abi(tmp_path, engine_lib):
    exe = tmp_path / "shim_test"
    lib_dir = ROOT / "mnrt_b200"
    r = subprocess.run([nvcc(), "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-L", str(lib_dir),
                        "-lpmgpu", "-Xlinker", f"-rpath,{lib_dir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim test ok" in r.stdout
