"""Builds the sm_100a shared library in-tree: aquarius_b200/libaquarius_b200.so.

    python -m aquarius_b200.build [--verbose]

nvcc compiles every csrc/*.cu for sm_100a only (no PTX fallback, no other
arch).  The CUDA runtime is linked statically, so the library carries no
dependency on a framework's CUDA runtime.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libaquarius_b200.so"
STAMP = PKG / ".libaquarius_b200.stamp"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", *ARCH,
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-shared", "-cudart", "static", "-Xlinker", "--no-undefined",
    f"-I{ROOT / 'include'}",
]


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def _digest() -> str:
    h = hashlib.sha256()
    for p in sorted(list(CSRC.glob("*")) + [ROOT / "include" / "aquarius_b200.h", pathlib.Path(__file__)]):
        if p.is_file():
            h.update(p.name.encode())
            h.update(p.read_bytes())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the library needs the CUDA toolkit to build")
    return exe


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    dig = _digest()
    if LIB.exists() and STAMP.exists() and STAMP.read_text() == dig and not force:
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose else []),
           *map(str, sources()), "-o", str(LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed building libaquarius_b200.so")
    STAMP.write_text(dig)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
