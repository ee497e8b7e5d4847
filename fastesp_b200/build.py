"""Compile libfastesp_b200.so in-tree for sm_100a.

    python -m fastesp_b200.build [--force]

The library is one nvcc translation unit (csrc/fastesp_b200.cu); the per-class
code in csrc/classes_gen.cuh is regenerated first when gen_classes.py or
hermite.py is newer than it.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libfastesp_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found (set NVCC)")


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + \
        [PKG.parents[0] / "include" / "fastesp_b200.h"]


def generate(force: bool = False) -> None:
    gen = CSRC / "classes_gen.cuh"
    deps = [CSRC / "gen_classes.py", PKG / "hermite.py"]
    if force or not gen.exists() or any(d.stat().st_mtime > gen.stat().st_mtime for d in deps):
        subprocess.run([sys.executable, str(CSRC / "gen_classes.py")], check=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    generate()
    if not force and LIB.exists() and all(s.stat().st_mtime <= LIB.stat().st_mtime
                                          for s in _sources()):
        return LIB
    tmp = LIB.with_suffix(f".so.tmp{os.getpid()}")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-o", str(tmp), str(CSRC / "fastesp_b200.cu")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-6000:])
    if verbose:
        print(r.stderr)
    (PKG / "ptxas.log").write_text(r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
