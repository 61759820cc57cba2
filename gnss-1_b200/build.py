"""Build recipe for libgnss_b200.so (sm_100a), in tree next to this file.

    python gnss-1_b200/build.py [--verbose-ptxas] [--force]

nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3, one shared
library exporting the C ABI of include/gnss_b200.h.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SOURCES = [HERE / "csrc" / "gnss_b200.cu", HERE / "csrc" / "batch.cpp", HERE / "csrc" / "io.cpp",
           HERE / "csrc" / "ic.cu"]
DEPS = sorted((HERE / "csrc").glob("*")) + [ROOT / "include" / "gnss_b200.h"]
OUT = HERE / "libgnss_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-shared", f"-I{ROOT / 'include'}"]


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in DEPS)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not verbose_ptxas and up_to_date():
        return OUT
    cmd = [NVCC, *FLAGS, "-o", str(OUT), *map(str, SOURCES)]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    p = build(a.force, a.verbose_ptxas)
    print(p)
    sys.exit(0)
