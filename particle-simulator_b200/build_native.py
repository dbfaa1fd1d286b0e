"""Build ``libdem_b200.so`` (the CUDA kernels and the C ABI) for sm_100a.

    python particle-simulator_b200/build_native.py [--force] [-v]

Each ``csrc/*.cu`` is compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a
-O3 -lineinfo``; the files whose results must be bit-identical to the
reference's expression order are compiled with ``-fmad=false`` (no implicit
multiply-add contraction).  The library is linked in-tree next to the ``dem``
package so that it travels with the checkout.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libdem_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          f"-I{INCLUDE}", f"-I{CSRC}", "-Xptxas", "-warn-spills"]
# reference-order FP64 arithmetic: no contraction
NO_FMAD = {"direct_fp64.cu", "euler.cu", "hash.cu", "merge.cu", "tree.cu"}
# FP32 pair terms never see denormal operands (r^2 >= (k (r_i + r_j))^2 on the
# FP32 path): flush-to-zero keeps rsqrtf and the FP32 ops to single instructions
FTZ = {"direct_mixed.cu", "direct_mixed_sym.cu"}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def _deps():
    return list(CSRC.glob("*.cuh")) + [INCLUDE / "dem_b200.h"]


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    newest_dep = max(p.stat().st_mtime for p in _deps() + [src, Path(__file__)])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    flags = list(COMMON)
    if src.name in NO_FMAD:
        flags.append("-fmad=false")
    if src.name in FTZ:
        flags.append("-ftz=true")
    if verbose:
        flags += ["-Xptxas", "-v"]
    cmd = [nvcc(), *ARCH, *flags, "-c", str(src), "-o", str(obj)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{p.stdout}\n{p.stderr}")
    if verbose and (p.stdout or p.stderr):
        print(f"--- {src.name}\n{p.stdout}{p.stderr}", file=sys.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if LIB.exists() and not force and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"link failed:\n{p.stdout}\n{p.stderr}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
