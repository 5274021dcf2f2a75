"""Builds the engine's shared library for sm_100a, in tree, and the
synthetic-input generator beside it.

    python -m jxr_b200.build          # -> jxr_b200/libjxr_b200.so, jxr_b200/libjxr_synth.so

nvcc cross-compiles without a GPU, so this runs anywhere the CUDA toolkit is
installed.  The engine library links the CUDA runtime statically and exports
the C ABI of include/jxr_b200.h.  The generator (csrc/synth.h: seeded images
coded by the forward half of the codec) is host code only and lives in a
library of its own, so that a process which only needs inputs -- the
benchmark's CPU reference arm -- never maps the engine.
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
SYNTH_LIB = PKG / "libjxr_synth.so"
SOURCES = ["recon_kernel.cu", "static_scratch.cu", "orient.cu", "analysis.cu", "host.cpp", "sample_scale.cpp"]
HEADERS = ["engine.h", "lifting.cuh", "forward.h", "sample_scale.h"]
SYNTH_SOURCES = ["synth.cpp"]
SYNTH_HEADERS = ["synth.h", "forward.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the engine")


def _stale(lib: Path, sources, headers) -> bool:
    if not lib.exists():
        return True
    built = lib.stat().st_mtime
    deps = [CSRC / s for s in list(sources) + list(headers)] + [ROOT / "include" / "jxr_b200.h", Path(__file__)]
    return any(d.exists() and d.stat().st_mtime > built for d in deps)


def build_synth(force: bool = False) -> Path:
    """The generator library: plain host C++ with OpenMP, through nvcc's host
    compiler (no device code, no CUDA runtime)."""
    if not force and not _stale(SYNTH_LIB, SYNTH_SOURCES, SYNTH_HEADERS):
        return SYNTH_LIB
    tmp = SYNTH_LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), "-O3", "-std=c++17", "-shared", "-cudart", "none", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC,-fopenmp",
                    "-I", str(ROOT / "include"), "-I", str(CSRC), *[str(CSRC / s) for s in SYNTH_SOURCES],
                    "-o", str(tmp)], check=True)
    os.replace(tmp, SYNTH_LIB)
    return SYNTH_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    build_synth(force)
    if not force and not _stale(LIB, SOURCES, HEADERS):
        return LIB
    out_dir = PKG / "_build"
    out_dir.mkdir(exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-I", str(CSRC)]
    for src in SOURCES:
        obj = out_dir / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", *common, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
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
    print(SYNTH_LIB)
