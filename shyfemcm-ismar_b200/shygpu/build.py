"""Build libshygpu.so (sm_100a) in-tree with nvcc.

    python shyfemcm-ismar_b200/shygpu/build.py [--verbose]

The library links only the CUDA runtime; its C ABI is include/shygpu.h.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = HERE / "libshygpu.so"
SOURCES = ["step_node32.cu", "step_node16.cu", "step_zeta.cu", "step_node.cu", "step.cu", "host.cu",
           "static_solve.cu", "serve.cu", "nonhydro.cu"]
HEADERS = ["common.cuh", "launch.h", "physics.cuh", "node_launch.cuh", "k_column.cuh", "k_column_t.cuh", "k_final.cuh", "k_node.cuh", "k_conz.cuh", "k_zeta.cuh", "k_wetdry.cuh", "k_zeta_global.cuh", "k_zeta_grid.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
    "-I", str(ROOT / "include"),
]


def nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "shygpu.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(verbose=False, force=False):
    if not force and not stale():
        return LIB
    objs, procs = [], []
    build_dir = PKG / "_build"
    build_dir.mkdir(exist_ok=True)
    for src in SOURCES:          # the translation units compile concurrently
        obj = build_dir / (Path(src).stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(str(obj))
    failed = [cmd for cmd, pr in procs if pr.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp),
           "-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
