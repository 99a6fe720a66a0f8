"""Builds libmcg.so in-tree for sm_100a (nvcc + the system g++).

Usage: python -m mcscram_b200.build [--force]

The library is a plain C ABI (include/mcg.h, include/mcg_host.h); no torch
types cross it.  Object files go to mcscram_b200/_build/ and the shared
library to mcscram_b200/libmcg.so, next to this file, so it travels with the
source tree.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libmcg.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
              "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmcg.so")
    return cand


def _cxx() -> str:
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _digest() -> str:
    h = hashlib.sha256()
    for p in sorted(list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))):
        if p.is_file():
            h.update(p.name.encode())
            h.update(p.read_bytes())
    h.update(" ".join(ARCH + NVCC_FLAGS + CXX_FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every CUDA/C++ source and links libmcg.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    stamp = BUILD / "digest"
    dig = _digest()
    if LIB.exists() and stamp.exists() and stamp.read_text() == dig and not force:
        return LIB
    nvcc, cxx = _nvcc(), _cxx()
    inc = [f"-I{INCLUDE}", f"-I{CSRC}"]
    objs = []
    procs = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        if src.suffix == ".cu":
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-ccbin", cxx, *inc, "-c", str(src), "-o", str(obj)]
        else:
            cmd = [cxx, *CXX_FLAGS, *inc, "-I/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
        procs.append((src, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = []
    for src, cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out))
        elif verbose and out:
            print(out)
    if failed:
        msg = "\n".join(f"--- {s.name}\n{o}" for s, o in failed)
        raise RuntimeError(f"libmcg build failed:\n{msg}")
    tmp = LIB.with_suffix(".so.tmp")
    link = [nvcc, *ARCH, "-shared", "-ccbin", cxx, "-o", str(tmp), *map(str, objs), "-cudart", "static",
            "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"libmcg link failed:\n{r.stdout}")
    os.replace(tmp, LIB)
    stamp.write_text(dig)
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(path)
