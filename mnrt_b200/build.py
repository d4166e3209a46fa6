"""Builds the engine's shared library (sm_100a) and the CPU oracle in-tree.

    python -m mnrt_b200.build          # engine + oracle
    python -m mnrt_b200.build --engine # engine only

The engine library lands at mnrt_b200/libpmgpu.so; the oracle (test
infrastructure) at oracle/_build/liboracle.so.  nvcc cross-compiles for
sm_100a without a GPU present.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libpmgpu.so"
SOURCES = ["pm_api.cu", "pm_build.cu", "pm_query.cu", "pm_sort.cu", "pm_backward.cu", "pm_gather.cu", "pm_batch.cu",
           "pm_compat.cu", "pm_icut.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the engine needs the CUDA toolkit to build")
    return cand


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_engine(force: bool = False, verbose: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "pmgpu.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared", "-o", str(LIB) + ".tmp",
           *map(str, srcs), "-I", str(ROOT / "include")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


def build_oracle(force: bool = False) -> Path:
    odir = ROOT / "oracle"
    out = odir / "_build" / "liboracle.so"
    if not force and not _stale(out, [odir / "pm_oracle.cpp"]):
        return out
    r = subprocess.run(["make", "-C", str(odir), "-B" if force else "all"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--engine", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build_engine(force=a.force, verbose=a.verbose))
    if not a.engine:
        print(build_oracle(force=a.force))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
