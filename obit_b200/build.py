"""Build libobit_dft.so in-tree for sm_100a.

nvcc compiles the CUDA sources (kernels, planner, C ABI) with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``; gcc compiles the C host
mirror of the GPU sky-model class; nvcc links them into
``obit_b200/libobit_dft.so`` (CUDA runtime linked statically).  Rebuilds only
when a source or header is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libobit_dft.so"
OBJ = PKG / "_build"

CU_SOURCES = ["dft_plan.cu", "dft_batch_kernels.cu", "dft_beam.cu", "dft_beam_mma.cu", "beam_jones.cu", "abi_layout.cu",
              "obit_dft_capi.cu", "obit_dft_static.cu", "dft_batch.cu", "grid_model.cu",
              "resident.cu"]
C_SOURCES = ["gpu_skymodel.c"]
CXX_SOURCES = ["dft_planner.cpp", "cc_loader.cpp", "grid_host.cpp", "subuv.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libobit_dft.so")


def _cuda_include() -> str:
    nvcc = Path(_nvcc()).resolve()
    return str(nvcc.parent.parent / "include")


def _inputs() -> list[Path]:
    files = [CSRC / s for s in CU_SOURCES + C_SOURCES + CXX_SOURCES]
    files += list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.inc")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    files.append(Path(__file__))
    return files


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in _inputs())


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return p.stdout + p.stderr


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile libobit_dft.so if needed and return its path."""
    if not force and up_to_date():
        return LIB
    OBJ.mkdir(exist_ok=True)
    nvcc = _nvcc()
    jobs = []
    for s in CU_SOURCES:
        cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               f"-I{INCLUDE}", "-c", str(CSRC / s), "-o", str(OBJ / (s + ".o"))]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        jobs.append(cmd)
    for s in C_SOURCES:
        jobs.append(["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", f"-I{INCLUDE}",
                     f"-I{_cuda_include()}", "-c", str(CSRC / s), "-o", str(OBJ / (s + ".o"))])
    for s in CXX_SOURCES:
        # no floating-point contraction: the component loader rounds where the
        # reference's single-precision code does
        jobs.append(["g++", "-O2", "-fPIC", "-std=c++17", "-Wall", "-ffp-contract=off", f"-I{INCLUDE}",
                     f"-I{_cuda_include()}", "-c", str(CSRC / s), "-o", str(OBJ / (s + ".o"))])
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        logs = list(ex.map(lambda c: _run(c, verbose), jobs))
    if ptxas_info:
        for log in logs:
            print(log, file=sys.stderr)
    objs = [str(OBJ / (s + ".o")) for s in CU_SOURCES + C_SOURCES + CXX_SOURCES]
    tmp = LIB.with_suffix(".so.tmp")
    # cuFFT (the gridded model's FFT) from the toolkit, found at run time where it lies
    cuda_lib = str(Path(_cuda_include()).parent / "lib64")
    _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, f"-L{cuda_lib}", "-lcufft",
          "-Xlinker", f"-rpath={cuda_lib}", "-lpthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Build the CPU oracles under oracle/ (test infrastructure)."""
    _run(["make", "-s", "-C", str(ROOT / "oracle")], verbose)


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True, ptxas_info="--ptxas" in sys.argv))
