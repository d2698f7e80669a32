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

Usage: python oracle/build_ref.py [reference_root]   (default /root/reference). Without the
reference sources the build is skipped and an existing library is kept.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libqhref.so"

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


def build(reference_root: str | os.PathLike = "/root/reference", force: bool = False) -> Path | None:
    root = Path(reference_root)
    if not (root / "src" / "api.cpp").exists():
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


if __name__ == "__main__":
    lib = build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", force=True)
    print(lib if lib else "reference sources absent; nothing built")
