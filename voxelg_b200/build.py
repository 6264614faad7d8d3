"""Build libvoxrt.so in-tree with nvcc for sm_100a.

Usage: python -m voxelg_b200.build [--force] [--no-checked]

The traversal and world kernels are compiled with --fmad=false and IEEE
divide/sqrt so that every float operation is a single IEEE binary32
operation in the reference's order (hit records must be bit-exact against
the CPU restatement).  Objects go to voxelg_b200/_build/, the library to
voxelg_b200/lib/libvoxrt.so.  The checked library (VX_CHECKED: every
world-array load of the traversal bounds-checked, vx_world_oob) is built
beside it from the same sources, objects in voxelg_b200/_build/checked/.
Translation units compile in parallel.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libvoxrt.so"
LIB_CHECKED = PKG / "lib" / "libvoxrt_checked.so"
# the chunk generator's powf / cosf / sinf exception table (vx_gmath.h),
# written beside the library for the C library this host runs
LMX_TABLE = PKG / "lib" / "vx_libm_exceptions.bin"
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
    ("vx_resident.cu", EXACT),
    ("vx_learned.cu", EXACT),
    ("vx_distfield.cu", []),
    ("vx_pack.cu", []),
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


def _build_lib(build_dir: Path, lib: Path, defines: list[str], force: bool,
               verbose: bool) -> Path:
    build_dir.mkdir(parents=True, exist_ok=True)
    lib.parent.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objs, cmds = [], []
    for name, extra in SOURCES:
        src = CSRC / name
        obj = build_dir / (name + ".o")
        objs.append(obj)
        if force or _newer(src, obj, headers):
            lang = ["-x", "cu"] if name.endswith(".cpp") else []
            cmds.append([nvcc(), *lang, *ARCH, *COMMON, *defines, *extra, "-c", str(src),
                         "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    if cmds:
        with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
            list(ex.map(run, cmds))
    if cmds or not lib.exists():
        tmp = lib.with_suffix(".so.tmp")
        run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static",
             "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"])
        os.replace(tmp, lib)
    return lib


def build_libm_table(force: bool = False, verbose: bool = False) -> Path:
    """vx_libm_exceptions.bin: compiles vx_libmx_gen.cpp for the host and runs
    it (an exhaustive scan of powf over [0, 1], about 20 s on 8 cores) when the
    table is missing or older than its sources."""
    src = CSRC / "vx_libmx_gen.cpp"
    deps = [src, CSRC / "vx_gmath.h"]
    if not force and LMX_TABLE.exists() and not _newer(src, LMX_TABLE, deps):
        return LMX_TABLE
    BUILD.mkdir(parents=True, exist_ok=True)
    LMX_TABLE.parent.mkdir(exist_ok=True)
    exe = BUILD / "vx_libmx_gen"
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-ffp-contract=off", "-std=c++17", "-pthread", f"-I{CSRC}", str(src), "-o",
           str(exe)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    tmp = LMX_TABLE.with_suffix(".bin.tmp")
    out = subprocess.run([str(exe), str(tmp)], check=True, capture_output=True, text=True)
    if verbose:
        print(out.stdout.strip(), flush=True)
    os.replace(tmp, LMX_TABLE)
    return LMX_TABLE


def build(force: bool = False, verbose: bool = False, checked: bool = True) -> Path:
    """libvoxrt.so, the checked library beside it unless checked=False, and
    the generator's math exception table."""
    jobs = [(BUILD, LIB, [])]
    if checked:
        jobs.append((BUILD / "checked", LIB_CHECKED, ["-DVX_CHECKED=1"]))
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        list(ex.map(lambda j: _build_lib(*j, force, verbose), jobs))
    build_libm_table(force, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, checked="--no-checked" not in sys.argv)
    print(LIB)
