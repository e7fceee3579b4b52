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
SOURCES = ["mcs_kernels.cu", "mcs_lobes.cu", "mcs_surrogate.cu", "mcs_probe.cu", "mcs_spindle.cpp",
           "mcs_engine.cu", "mcs_api.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists() and not shutil.which(cand):
        raise RuntimeError("nvcc not found")
    return cand


BUILD = HERE / "_build"
# (source, object, extra flags): the kernels file builds once per integration precision
UNITS = [("mcs_kernels.cu", "mcs_kernels_f32.o", ["-DMCS_PREC=32"]),
         ("mcs_kernels.cu", "mcs_kernels_f64.o", ["-DMCS_PREC=64"]),
         ("mcs_lobes.cu", "mcs_lobes.o", []),
         ("mcs_surrogate.cu", "mcs_surrogate.o", []),
         ("mcs_probe.cu", "mcs_probe.o", []),
         ("mcs_spindle.cpp", "mcs_spindle.o", []),
         # separately rounded products and sums, as the reference's JavaScript evaluates
         ("mcs_engine.cu", "mcs_engine.o", ["-fmad=false"]),
         ("mcs_api.cu", "mcs_api.o", [])]


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + [ROOT / "include" / "mcs.h"]
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> Path:
    """Compile every unit to an object in parallel, then link libmcs.so."""
    if not force and not needs_build():
        return OUT
    BUILD.mkdir(exist_ok=True)
    nvc = nvcc()
    base = [nvc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
            "-Xcompiler", "-Wall", "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]
    if verbose_ptxas:
        base += ["-Xptxas", "-v"]
    procs = []
    for src, obj, extra in UNITS:
        cmd = base + extra + ["-c", str(CSRC / src), "-o", str(BUILD / obj)]
        print(" ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd))
    bad = [u for u, p in zip(UNITS, procs) if p.wait() != 0]
    if bad:
        raise RuntimeError(f"nvcc failed on {[u[0] for u in bad]}")
    link = [nvc, *ARCH, "-shared", "-o", str(OUT)] + [str(BUILD / u[1]) for u in UNITS]
    link += ["-lcudart"]
    print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
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
