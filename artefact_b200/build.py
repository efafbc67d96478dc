"""Build the native library of artefact_b200 in-tree.

Compiles the CUDA kernels and the host C ABI for sm_100a with nvcc into
``artefact_b200/libartefact_b200.so`` (static CUDA runtime, no torch
dependency). Run as ``python -m artefact_b200.build`` or through
``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libartefact_b200.so"

SOURCES = ["solver.cu", "cnn.cu", "capi_host.cpp", "jpeg_decode.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build artefact_b200")
    return exe


def _stale() -> bool:
    if not LIB.exists():
        return True
    mtime = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > mtime for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if a source is newer than it; return its path."""
    if not force and not _stale():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [
        nvcc(), *GENCODE, "-lineinfo", "-O3", "-std=c++17", "-shared",
        "-Xcompiler", "-fPIC,-O2", "-Xptxas", "-v" if verbose else "-O3",
        "-I", str(INCLUDE), "-o", str(tmp),
        *[str(CSRC / s) for s in SOURCES],
    ]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(res.stderr, file=sys.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
