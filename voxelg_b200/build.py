"""Build libvoxrt.so in-tree with nvcc for sm_100a.

Usage: python -m voxelg_b200.build [--force]

The traversal and world kernels are compiled with --fmad=false and IEEE
divide/sqrt so that every float operation is a single IEEE binary32
operation in the reference's order (hit records must be bit-exact against
the CPU restatement).  Objects go to voxelg_b200/_build/, the library to
voxelg_b200/lib/libvoxrt.so.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libvoxrt.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# exact IEEE binary32: no contraction, no flush-to-zero, IEEE div/sqrt
EXACT = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
          f"-I{INCLUDE}", f"-I{CSRC}"]

# (source, extra flags)
SOURCES = [
    ("vx_trace.cu", EXACT),
    ("vx_world.cu", EXACT),
    ("vx_slotgen.cu", EXACT),
    ("vx_noalloc.cu", EXACT),
    ("vx_queue.cu", EXACT),
    ("vx_learned.cu", EXACT),
    # the proposal network: its values only steer the verified restart
    ("vx_mlp.cu", []),
    ("vx_proposal.cpp", []),
    ("vx_api.cpp", []),
    ("vx_host_world.cpp", []),
    ("vx_serve.cpp", []),
    ("vx_wire.cpp", []),
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _newer(src: Path, dst: Path, deps: list[Path]) -> bool:
    if not dst.exists():
        return True
    t = dst.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objs = []
    changed = force
    for name, extra in SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if force or _newer(src, obj, headers):
            cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
            if name.endswith(".cpp"):
                cmd = [nvcc(), "-x", "cu", *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            changed = True
    if changed or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static",
               "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
