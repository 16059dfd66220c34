"""Build libpfa_b200.so for sm_100a with nvcc (in-tree; the .so travels with the checkout).

    python mpfs250t-sar-ifp_b200/build.py            # incremental
    python mpfs250t-sar-ifp_b200/build.py --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "pfa_b200" / "lib" / "libpfa_b200.so"
BUILD = PKG / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]
SOURCES = ["pfa_capi.cu", "pfa_fixed.cu", "pfa_float.cu", "pfa_mixed.cu", "pfa_noalloc.cu", "pfa_display.cu"]


def _gen():
    sys.path.insert(0, str(PKG))
    from pfa_b200 import tables
    tables.write_c_include(CSRC / "gen" / "sinc_q15.inc")


def _newer(src: Path, deps, dst: Path) -> bool:
    if not dst.exists():
        return True
    t = dst.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> Path:
    _gen()
    BUILD.mkdir(exist_ok=True)
    OUT.parent.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((CSRC / "gen").glob("*.inc")) + \
        [PKG.parent / "include" / "pfa_b200.h"]
    objs = []
    for s in SOURCES:
        src = CSRC / s
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _newer(src, headers, obj):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_v:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or any(_newer(o, [], OUT) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(OUT), *map(str, objs)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.v, a.ptxas_v))
