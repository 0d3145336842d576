"""Build the sm_100a shared library anelastic_solve_b200/libanel.so with nvcc.

Each .cu file compiles to its own object (in parallel), then one nvcc link
step makes the shared library.  The FP64 parity-critical files are compiled
with ``-fmad=false`` (no multiply-add contraction) and the host compiler
with ``-ffp-contract=off``; the FP32 inner-cycle file keeps FMA.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libanel.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
          "-ffp-contract=off", "--expt-relaxed-constexpr", "-I", str(CSRC)]
# file -> extra flags
SOURCES = {
    "api.cu": ["-fmad=false"],
    "mg_solver.cu": ["-fmad=false"],
    "mg_kernels64.cu": ["-fmad=false"],
    "mg_kernels32.cu": ["-fmad=true"],
    "ns_kernels.cu": ["-fmad=false"],
    "ns_solver.cu": ["-fmad=false"],
    "noalloc.cu": ["-fmad=false"],
    "serve.cu": ["-fmad=false"],
    "restart.cu": ["-fmad=false"],
    "ns_dsm.cu": ["-fmad=false"],
    "mg_col.cu": ["-fmad=true"],
    "mg_col64.cu": ["-fmad=false"],
    "tune.cu": [],
    "mg_coarse.cu": ["-fmad=true"],
}


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _compile(src: str, flags: list[str], verbose: bool) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    srcp = CSRC / src
    deps = [srcp] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [
        PKG.parent / "include" / "anel.h"]
    if obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(srcp), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), SOURCES.items()))
    if LIB.exists() and not force and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
