"""Build libvocalsim_b200.so in-tree (lib/) for sm_100a with nvcc.

    python vocalsim-2p5d-fdtd_b200/build.py [--force]

Host C++ is compiled with -ffp-contract=off so the map builder rounds every
float operation separately, like the reference's x86-64 host build; device
code uses explicit round-to-nearest intrinsics and --fmad=false.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib" / "libvocalsim_b200.so"
OBJ = PKG / "_build"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
              f"-I{INCLUDE}", "-Wno-deprecated-gpu-targets"]

SOURCES = ["vs_grid.cpp", "vs_capi.cpp", "vs_step.cu", "vs_cluster.cu", "vs_noalloc.cu", "vs_adjoint.cu", "vs_mapbuild.cu", "vs_spectrum.cu",
           "vs_sections.cu", "vs_audio.cu", "vs_shapes.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "vocalsim_b200.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            lang = ["-x", "cu"] if s.suffix == ".cu" else ["-x", "c++"]
            cmd = [nvcc(), *NVCC_FLAGS, *ARCH, *lang, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        # cuFFT (vs_formants) is linked dynamically from the toolkit next to nvcc
        cuda_lib = Path(nvcc()).resolve().parent.parent / "lib64"
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-ldl", "-lrt",
               "-lpthread", f"-L{cuda_lib}", "-lcufft", "-Xlinker", f"-rpath={cuda_lib}"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
