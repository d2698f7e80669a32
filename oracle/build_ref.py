"""Builds oracle/_ref/libqhref.so: the reference's own CPU implementation, compiled unmodified
from its sources where they lie, plus the flat C wrapper in oracle/ref_capi.cpp.

Test infrastructure only. The reference's CMake build fetches pocketfft, googletest and nanobind
from the network; none of that is needed here. The library is compiled directly with g++ from:

  src/api.cpp src/pipeline.cpp src/bpm.cpp src/phantom.cpp
  src/cpu/fft.cpp src/cpu/field.cpp src/cpu/unwrap.cpp src/cpu/odt.cpp src/cpu/tv.cpp src/cpu/bpm.cpp

with oracle/pocketfft_shim standing in for the absent pocketfft header (the only third-party code
those sources include; used by src/cpu/fft.cpp:9-66). Flags: -std=c++20 -O2 -fopenmp
-ffp-contract=off and no -march=native, so the host float arithmetic of the Ewald mapping
(src/common.hpp:56-67) is evaluated unfused, as on a stock x86-64 build.

A second library, oracle/_ref/libqhref_cuda.so, adds the reference's CUDA backend: the same sources
with QORAHOLO_HAS_CUDA defined (as the reference's CMake option QORAHOLO_CUDA does) plus
src/cuda/{runtime,field,unwrap,bpm,odt,tv,pipeline}.cu compiled unmodified by nvcc for sm_100a and
linked against cudart and cuFFT -- the reference's own GPU path, timed on the same B200 as the bar
for this project's kernels. It is built only where nvcc is present.

Usage: python oracle/build_ref.py [reference_root]. The reference root is the argument, else the
QORAHOLO_REFERENCE environment variable. Without the reference sources the build is skipped and
existing libraries are kept.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libqhref.so"
LIB_CUDA = OUT_DIR / "libqhref_cuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_SOURCES = ["src/cuda/runtime.cu", "src/cuda/field.cu", "src/cuda/unwrap.cu", "src/cuda/bpm.cu",
                "src/cuda/odt.cu", "src/cuda/tv.cu", "src/cuda/pipeline.cu"]


def reference_root(arg=None) -> Path | None:
    """The reference checkout: the argument, else $QORAHOLO_REFERENCE; None when neither is set."""
    root = arg or os.environ.get("QORAHOLO_REFERENCE")
    return Path(root) if root else None

SOURCES = [
    "src/api.cpp",
    "src/pipeline.cpp",
    "src/bpm.cpp",
    "src/phantom.cpp",
    "src/cpu/fft.cpp",
    "src/cpu/field.cpp",
    "src/cpu/unwrap.cpp",
    "src/cpu/odt.cpp",
    "src/cpu/tv.cpp",
    "src/cpu/bpm.cpp",
]


def build(root: str | os.PathLike | None = None, force: bool = False) -> Path | None:
    root = reference_root(root)
    if root is None or not (root / "src" / "api.cpp").exists():
        return LIB if LIB.exists() else None
    OUT_DIR.mkdir(exist_ok=True)
    inputs = [root / s for s in SOURCES] + [HERE / "ref_capi.cpp", HERE / "pocketfft_shim" / "pocketfft_hdronly.h"]
    if LIB.exists() and not force:
        newest = max(p.stat().st_mtime for p in inputs)
        if LIB.stat().st_mtime >= newest:
            return LIB
    objs = []
    flags = ["-std=c++20", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC",
             f"-I{root / 'include'}", f"-I{root / 'src'}", f"-I{HERE / 'pocketfft_shim'}"]
    jobs = []
    for src in inputs[:-1]:
        obj = OUT_DIR / (src.stem + ("_ref" if src.parent.name == "cpu" else "") + ".o")
        if src.parent.name == "cpu":
            obj = OUT_DIR / ("cpu_" + src.stem + ".o")
        objs.append(obj)
        jobs.append(subprocess.Popen(["g++", *flags, "-c", str(src), "-o", str(obj)]))
    for j in jobs:
        if j.wait() != 0:
            raise RuntimeError("oracle/_ref build failed")
    subprocess.check_call(["g++", "-shared", "-fopenmp", "-o", str(LIB), *map(str, objs)])
    for o in objs:
        o.unlink()
    return LIB


def build_cuda(root: str | os.PathLike | None = None, force: bool = False) -> Path | None:
    """The reference with its CUDA backend (libqhref_cuda.so); None without sources or nvcc."""
    root = reference_root(root)
    if root is None or not (root / "src" / "cuda" / "odt.cu").exists() or not Path(NVCC).exists():
        return LIB_CUDA if LIB_CUDA.exists() else None
    OUT_DIR.mkdir(exist_ok=True)
    cxx_inputs = [root / s for s in SOURCES] + [HERE / "ref_capi.cpp"]
    cu_inputs = [root / s for s in CUDA_SOURCES]
    deps = cxx_inputs + cu_inputs + [HERE / "pocketfft_shim" / "pocketfft_hdronly.h"]
    if LIB_CUDA.exists() and not force and LIB_CUDA.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return LIB_CUDA
    cuda_inc = Path(NVCC).resolve().parent.parent / "include"
    cuda_lib = Path(NVCC).resolve().parent.parent / "lib64"
    inc = [f"-I{root / 'include'}", f"-I{root / 'src'}", f"-I{HERE / 'pocketfft_shim'}"]
    objs, jobs = [], []
    for src in cxx_inputs:
        obj = OUT_DIR / ("cu_" + ("cpu_" if src.parent.name == "cpu" else "") + src.stem + ".o")
        objs.append(obj)
        jobs.append(subprocess.Popen(["g++", "-std=c++20", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC",
                                      "-DQORAHOLO_HAS_CUDA", f"-I{cuda_inc}", *inc, "-c", str(src), "-o", str(obj)]))
    for src in cu_inputs:
        obj = OUT_DIR / ("cu_dev_" + src.stem + ".o")
        objs.append(obj)
        jobs.append(subprocess.Popen([NVCC, "-std=c++20", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                                      "-Xcompiler", "-fPIC", "-DQORAHOLO_HAS_CUDA", *inc, "-c", str(src), "-o",
                                      str(obj)]))
    for j in jobs:
        if j.wait() != 0:
            raise RuntimeError("oracle/_ref CUDA build failed")
    subprocess.check_call(["g++", "-shared", "-fopenmp", "-o", str(LIB_CUDA), *map(str, objs), f"-L{cuda_lib}",
                           "-lcufft", "-lcudart", f"-Wl,-rpath,{cuda_lib}"])
    for o in objs:
        o.unlink()
    return LIB_CUDA


if __name__ == "__main__":
    arg = sys.argv[1] if len(sys.argv) > 1 else None
    lib = build(arg, force=True)
    print(lib if lib else "reference sources absent; nothing built")
    lib = build_cuda(arg, force=True)
    print(lib if lib else "reference CUDA backend not built (no sources or no nvcc)")
