"""Build recipe of the CUDA library libinmsom_gpu.so (sm_100a only).

The library is built in-tree, next to this file, so that it travels with
the repository.  general.cu and column.cu are compiled with --fmad=false
(per-loop and per-column kernels that round exactly like the Fortran
expressions); the fused streaming
kernel and the C ABI layer use the default contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libinmsom_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}"]
SOURCES = {
    "general.cu": ["--fmad=false"],
    "fused.cu": [],
    "capi.cu": [],
    "capi_column.cu": [],
    "capi_io.cu": [],
    "noalloc.cu": [],
    "closure.cu": [],
    "closure_tc.cu": [],
    "column.cu": ["--fmad=false"],
    "dstd.cu": [],
    "ctl_read.cu": [],
    "ocean_cp.cu": [],
}
HEADERS = ["common.cuh", "general.h", "fused.h", "closure.h", "column.h", "context.h", "gelu.cuh"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA source for sm_100a and link the shared library."""
    BUILD.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [INCLUDE / "inmsom_gpu.h"]
    objs = []
    for src, extra in SOURCES.items():
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src, *hdrs]):
            cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
