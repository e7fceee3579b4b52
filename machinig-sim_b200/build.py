"""Build libmcs.so in-tree with nvcc for sm_100a.

    python machinig-sim_b200/build.py [--verbose-ptxas]

The library has no PyTorch dependency: it is the C ABI of include/mcs.h over the CUDA
runtime, loaded by the Python host layer (ctypes) and the Node addon.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
OUT = HERE / "libmcs.so"
SOURCES = ["mcs_kernels.cu", "mcs_lobes.cu", "mcs_surrogate.cu", "mcs_api.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists() and not shutil.which(cand):
        raise RuntimeError("nvcc not found")
    return cand


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + [ROOT / "include" / "mcs.h"]
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> Path:
    if not force and not needs_build():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", "--expt-relaxed-constexpr", "-I", str(ROOT / "include"),
           "-o", str(OUT)]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(CSRC / s) for s in SOURCES]
    cmd += ["-lcudart"]
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    build(a.verbose_ptxas, a.force or a.verbose_ptxas)
    return 0


if __name__ == "__main__":
    sys.exit(main())
