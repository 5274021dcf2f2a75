"""Builds the engine's shared library for sm_100a, in tree.

    python -m jxr_b200.build          # -> jxr_b200/libjxr_b200.so

nvcc cross-compiles without a GPU, so this runs anywhere the CUDA toolkit is
installed.  The library links the CUDA runtime statically and exports the C ABI
of include/jxr_b200.h.
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
LIB = PKG / "libjxr_b200.so"
SOURCES = ["recon_kernel.cu", "static_scratch.cu", "host.cpp", "synth.cpp", "sample_scale.cpp"]
HEADERS = ["engine.h", "lifting.cuh", "synth.h", "forward.h", "sample_scale.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the engine")


def _stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "jxr_b200.h", Path(__file__)]
    return any(d.exists() and d.stat().st_mtime > built for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    out_dir = PKG / "_build"
    out_dir.mkdir(exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-I", str(CSRC)]
    for src in SOURCES:
        obj = out_dir / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", *common, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "cu"] if src.endswith(".cu") else []
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs,
                    "-Xcompiler", "-fopenmp"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
