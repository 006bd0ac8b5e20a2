"""Build librrtmg_b200.so for sm_100a (nvcc; no GPU needed) and the table blob.

Arithmetic flags are part of the numerics contract: -fmad=false keeps every
multiply and add a separate IEEE binary32 operation (the reference's WRF REAL
rounding), -prec-div/-prec-sqrt give correctly rounded division and square
root, and the host side is compiled without floating-point contraction.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "librrtmg_b200.so"
SOURCES = ("rrtmg_capi.cu", "rrtmg_mcica.cu", "rrtmg_lw.cu", "rrtmg_sw.cu", "surrogate_gemm.cu",
           "surrogate_ops.cu", "surrogate_capi.cu", "surrogate_mlp.cu", "rrtmg_prologue.cu",
           "rrtmg_tendency.cu", "rrtmg_tables.cu", "rrtmg_status.cu", "rrtmg_ffi.cu")
HEADERS = ("rrtmg_device.cuh", "rrtmg_kernels.h", "surrogate_kernels.h", "umma_common.cuh", "kiss_jump_host.h",
           "xla_ffi_abi.h")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-fmad=false",
              "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
              "-Xcompiler", "-fPIC,-ffp-contract=off"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile the CUDA sources (in parallel) and link librrtmg_b200.so."""
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [HERE.parent / "include" / "rrtmg_b200.h",
                                             HERE.parent / "include" / "rrtmg_surrogate.h",
                                             HERE.parent / "include" / "rrtmg_prologue.h",
                                             HERE.parent / "include" / "rrtmg_tendency.h",
                                             HERE.parent / "include" / "rrtmg_tables.h",
                                             HERE.parent / "include" / "rrtmg_xla_ffi.h"]
    objs = []
    jobs = []
    for src in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src, *headers]):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(run, jobs))
    if verbose:
        for log in logs:
            print(log)
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        run(cmd)
    return LIB


def main() -> None:
    import sys
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)


if __name__ == "__main__":
    main()
