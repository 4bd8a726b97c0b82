"""Compile the engine into chatcarlo_b200/lib/libccb200.so (FP32 tracking)
and libccb200_fp64.so (the same source tracking in FP64, the precision
reference), and the learned denoiser's kernels into
chatcarlo_b200/lib/libccunet.so (sm_100a).

``python -m chatcarlo_b200.build`` rebuilds a library when one of its
sources is newer than it.  The libraries link the CUDA runtime statically so
they load on any box with a driver, independent of the toolkit's library
path.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB_PATH = LIB_DIR / "libccb200.so"
HEADER = PKG.parent / "include" / "chatcarlo_b200.h"
SOURCES = [CSRC / "cc_engine.cu", CSRC / "cc_atomics.cu"]
DEPS = SOURCES + [CSRC / "philox.cuh", HEADER]
FP64_LIB_PATH = LIB_DIR / "libccb200_fp64.so"
UNET_LIB_PATH = LIB_DIR / "libccunet.so"
UNET_SOURCES = [CSRC / "cc_unet.cu"]
UNET_DEPS = UNET_SOURCES + [PKG.parent / "include" / "chatcarlo_b200_unet.h"]

# --use_fast_math: FP32 tracking tolerates approximate division, square root and
# transcendentals (the surface band is 8 ulps of the world extent); tallies are
# FP64 atomics of FP32 products either way.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "--use_fast_math", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static"]


# the precision reference: the engine tracking and sampling in FP64 with FP64
# tables and IEEE arithmetic (no fast-math intrinsics; more registers per
# thread, so two blocks per SM)
FP64_NVCC_FLAGS = [f for f in NVCC_FLAGS if f != "--use_fast_math"] + ["-DCC_TRACK_FP64", "-DCC_MIN_BLOCKS=2"]

# the denoiser's kernels keep IEEE arithmetic (their gradients are checked
# against an FP64 oracle)
UNET_NVCC_FLAGS = [f for f in NVCC_FLAGS if f != "--use_fast_math"]


def nvcc_path() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(lib: Path, deps: list[Path]) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def needs_build() -> bool:
    return _stale(LIB_PATH, DEPS) or _stale(FP64_LIB_PATH, DEPS) or _stale(UNET_LIB_PATH, UNET_DEPS)


def _compile(lib: Path, sources: list[Path], flags: list[str], verbose: bool) -> None:
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc_path(), *flags, "-o", str(tmp), *map(str, sources)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(res.stderr)
    os.replace(tmp, lib)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Build both libraries where stale; returns the engine's path."""
    if force or _stale(LIB_PATH, DEPS):
        _compile(LIB_PATH, SOURCES, NVCC_FLAGS, verbose)
    if force or _stale(FP64_LIB_PATH, DEPS):
        _compile(FP64_LIB_PATH, SOURCES, FP64_NVCC_FLAGS, verbose)
    if force or _stale(UNET_LIB_PATH, UNET_DEPS):
        _compile(UNET_LIB_PATH, UNET_SOURCES, UNET_NVCC_FLAGS, verbose)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
    print(FP64_LIB_PATH)
    print(UNET_LIB_PATH)
