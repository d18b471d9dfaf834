"""Build recipe of the in-tree CUDA library (sm_100a only).

    python -m waltz_b200.build        # -> waltz_b200/libwaltz_b200.so

The library is compiled with explicit fused multiply-adds only
(--fmad=false), IEEE division/square root and no flush-to-zero, because the
archives must be bit-identical to the reference CPU codec.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libwaltz_b200.so"
SOURCES = ["codec.cu", "cxx_api.cu"]
# HDF5 filter plugin (filter 61197), a separate library linked to LIB.
PLUGIN = PKG / "plugins" / "libwaltz_h5z.so"
PLUGIN_SOURCES = ["h5z_filter.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-ftz=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-O2", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise FileNotFoundError("nvcc not found")
    return path


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    deps = [CSRC / s for s in sources] + list(CSRC.glob("*.cuh")) + list((PKG.parent / "include").glob("*.h*"))
    return max(p.stat().st_mtime for p in deps) > target.stat().st_mtime


def build(force: bool = False, verbose: bool = False) -> Path:
    if force or _stale(LIB, SOURCES):
        srcs = [str(CSRC / s) for s in SOURCES]
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-o", str(tmp), *srcs]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    if force or _stale(PLUGIN, PLUGIN_SOURCES) or PLUGIN.stat().st_mtime < LIB.stat().st_mtime:
        PLUGIN.parent.mkdir(exist_ok=True)
        tmp = PLUGIN.with_suffix(".so.tmp")
        cmd = [nvcc(), *NVCC_FLAGS, "-o", str(tmp), *[str(CSRC / s) for s in PLUGIN_SOURCES],
               f"-L{PKG}", "-lwaltz_b200", "-Xlinker", "-rpath,$ORIGIN/.."]
        subprocess.run(cmd, check=True)
        os.replace(tmp, PLUGIN)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
