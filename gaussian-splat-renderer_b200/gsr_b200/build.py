"""Build recipe of the CUDA library libgsr_b200.so (sm_100a), in-tree.

    python -m gsr_b200.build            # from gaussian-splat-renderer_b200/
    python gaussian-splat-renderer_b200/gsr_b200/build.py [--force] [--verbose]

Steps: (1) compile and run csrc/gen_logf_fixups.c, which tabulates where this machine's C
library logf differs from the correctly rounded log on [1, 255]; (2) nvcc every .cu for
sm_100a (the bit-exact units with -fmad=false); (3) the host renderer with g++; (4) link one
shared library with the static CUDA runtime. Objects go to gaussian-splat-renderer_b200/_build/.
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
ROOT = PKG.parent  # gaussian-splat-renderer_b200/
REPO = ROOT.parent
CSRC = ROOT / "csrc"
INCLUDE = REPO / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libgsr_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}"]
# translation units whose floating-point results must match the reference bit for bit
# (the rasterizer's image is held to a tolerance instead and uses FMA and the hardware exp2)
EXACT_UNITS = {"k_front.cu", "k_encode.cu"}
CU_UNITS = ["k_front.cu", "k_sort.cu", "k_render.cu", "k_encode.cu", "k_mlp.cu"]
HOST_UNITS = ["renderer.cpp", "ply_loader.cpp", "training_cameras.cpp", "scene_io_abi.cpp", "color_checkpoint.cpp"]


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cpp"))
                  + list(CSRC.glob("*.c")) + [INCLUDE / "gsr_b200.h", Path(__file__)])


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    if not force and not stale():
        return LIB
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(parents=True, exist_ok=True)
    # (1) the logf fixup table, from this machine's C library
    gen = BUILD / "gen_logf_fixups"
    _run(["gcc", "-O2", "-ffp-contract=off", "-o", gen, CSRC / "gen_logf_fixups.c", "-lm"], verbose)
    table_c = BUILD / "logf_fixups.c"
    _run([gen, table_c], verbose)
    jobs = [(["gcc", "-O1", "-fPIC", "-c", table_c, "-o", BUILD / "logf_fixups.o"]), ]
    # (2) CUDA units
    for u in CU_UNITS:
        flags = ["-fmad=false"] if u in EXACT_UNITS else []
        if ptxas_info:
            flags += ["-Xptxas", "-v"]
        jobs.append([NVCC, *ARCH, *NVCC_COMMON, *flags, "-c", CSRC / u, "-o", BUILD / (u + ".o")])
    # (3) host units
    for u in HOST_UNITS:
        jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}",
                     f"-I{CUDA_HOME / 'include'}", "-c", CSRC / u, "-o", BUILD / (u + ".o")])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        outs = list(ex.map(lambda c: _run(c, verbose), jobs))
    if ptxas_info:
        for o in outs:
            if o.strip():
                print(o)
    # (4) link
    objs = [BUILD / "logf_fixups.o"] + [BUILD / (u + ".o") for u in CU_UNITS + HOST_UNITS]
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lpthread", "-ldl", "-lrt"], verbose)
    shutil.move(str(tmp), str(LIB))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force or args.ptxas_info, verbose=args.verbose, ptxas_info=args.ptxas_info))
    sys.exit(0)
