"""Ahead-of-time build of the sm_100a CUDA library ``libwrfgpu.so`` (in-tree).

The fp64 kernels are compiled with ``-fmad=false`` so their arithmetic keeps
the unfused operation order of the reference's float64 code.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libwrfgpu.so"
SELFTEST_LIB = HERE / "libwrfgpu_selftest.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build wrf_gpu_b200")
    return cand


def sources() -> list[Path]:
    return [CSRC / "dycore.cu"]


# (output library, its sources).  The self-test library holds device checks
# of numerical helpers that only the tests load.
TARGETS = ((LIB, [CSRC / "dycore.cu"]), (SELFTEST_LIB, [CSRC / "selftest.cu"]))


def _stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "wrfgpu.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile ``libwrfgpu.so`` (and the self-test library) for sm_100a if any
    source is newer than it."""
    for lib, srcs in TARGETS:
        if not force and not _stale(lib):
            continue
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
               "-I", str(HERE.parent / "include"), "-o", str(lib) + ".tmp", *map(str, srcs)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(str(lib) + ".tmp", lib)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
