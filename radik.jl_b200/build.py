"""Build libradik_b200.so (in-tree) with nvcc for sm_100a.

    python radik.jl_b200/build.py [--force] [--ptxas-verbose]

The library is the C ABI declared in include/radik.h.  The CUDA runtime is
linked statically (nvcc's default), so the .so only needs the NVIDIA driver.
"""
from __future__ import annotations

import argparse
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libradik_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build radik.jl_b200")


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def deps() -> list[pathlib.Path]:
    """Every file the library is compiled from: the .cu sources, their
    headers and the .inl files they include (the request server)."""
    return (sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inl"))
            + [ROOT / "include" / "radik.h"])


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps())


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> pathlib.Path:
    if not force and not stale():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-o", str(LIB)]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(s) for s in sources()]
    # The image exports CC/CXX pointing at a partial gcc; nvcc picks the host
    # compiler from PATH unless -ccbin is given.
    host_cxx = shutil.which("g++")
    if host_cxx:
        cmd[1:1] = ["-ccbin", host_cxx]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed ({res.returncode})")
    if not quiet or ptxas_verbose:
        sys.stderr.write(res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_verbose, quiet=False))
