"""In-tree build of the native libraries, for sm_100a (B200):

  qoraholo_b200/libqhk.so        CUDA kernels and the C ABI (include/qoraholo_b200.h)
  qoraholo_b200/libqoraholo.so   the C++20 host API (include/qoraholo/*.hpp) over the C ABI
  qoraholo_b200/_core*.so        pybind11 bindings with the reference's Python signatures

nvcc cross-compiles without a GPU. Objects go to qoraholo_b200/_build/; a library is rebuilt
when any of its sources or headers is newer. Usage: python qoraholo_b200/_build.py [--force] [--debug]
(run as a script: importing the package itself needs the built extension).

--debug also builds qoraholo_b200/debug/libqhk.so, the same ABI with the device bounds checks of
csrc/debug.cuh compiled in (QHK_DEBUG): the units that include debug.cuh are compiled again into
qoraholo_b200/_build_debug/, the others are linked from the release objects. Load it in place of the
release library with QHK_LIBRARY=qoraholo_b200/debug/libqhk.so (qoraholo_b200.capi).
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = ROOT / "include"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++20", "-O3", *ARCH, "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler",
              "-fPIC,-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}"]

LIB_QHK = PKG / "libqhk.so"
LIB_HOST = PKG / "libqoraholo.so"
BUILD_DEBUG = PKG / "_build_debug"
LIB_QHK_DEBUG = PKG / "debug" / "libqhk.so"


def _newest(paths):
    return max((p.stat().st_mtime for p in paths if p.exists()), default=0.0)


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(INCLUDE.rglob("*.h*"))


def _stale(obj: Path, src: Path) -> bool:
    """True when obj must be rebuilt: it or its dependency list (obj.d, written by the compiler's -MD
    -MF) is missing, or the source or any header it included is newer."""
    dep = obj.with_suffix(".d")
    if not obj.exists() or not dep.exists():
        return True
    text = dep.read_text().replace("\\\n", " ")
    files = [Path(t) for t in text.partition(":")[2].split()]
    built = obj.stat().st_mtime
    return any(not f.exists() or f.stat().st_mtime > built for f in [src, *files])


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    return r


def _compile(cmd):
    """One compile job; an object whose source or headers changed while it compiled is dated back to the
    start of the compile, so that the next build compiles it again."""
    t0 = time.time()
    _run(cmd)
    obj = Path(cmd[cmd.index("-o") + 1])
    dep = obj.with_suffix(".d")
    if dep.exists():
        files = [Path(t) for t in dep.read_text().replace("\\\n", " ").partition(":")[2].split()]
        if any(f.exists() and f.stat().st_mtime > t0 for f in files):
            os.utime(obj, (t0 - 1, t0 - 1))


def _compile_many(jobs):
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(_compile, jobs))


def build_qhk(force=False) -> Path:
    sources = sorted(CSRC.glob("*.cu"))
    BUILD.mkdir(exist_ok=True)
    jobs, objs = [], []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append([NVCC, *NVCC_FLAGS, "-MD", "-MF", str(obj.with_suffix(".d")), "-c", str(src), "-o", str(obj)])
    _compile_many(jobs)
    if force or jobs or not LIB_QHK.exists() or LIB_QHK.stat().st_mtime < _newest(objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB_QHK), *map(str, objs)])
    return LIB_QHK


def _uses_debug_checks(obj: Path) -> bool:
    """True when the release object's dependency list names debug.cuh (its unit has bounds checks)."""
    dep = obj.with_suffix(".d")
    return dep.exists() and "debug.cuh" in dep.read_text()


def build_qhk_debug(force=False) -> Path:
    """The debug library: the release objects, with the units that include debug.cuh recompiled with
    QHK_DEBUG."""
    build_qhk(False)
    BUILD_DEBUG.mkdir(exist_ok=True)
    LIB_QHK_DEBUG.parent.mkdir(exist_ok=True)
    jobs, objs = [], []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        if _uses_debug_checks(obj):
            obj = BUILD_DEBUG / (src.stem + ".o")
            if force or _stale(obj, src):
                jobs.append([NVCC, *NVCC_FLAGS, "-DQHK_DEBUG", "-MD", "-MF", str(obj.with_suffix(".d")), "-c",
                             str(src), "-o", str(obj)])
        objs.append(obj)
    _compile_many(jobs)
    if force or jobs or not LIB_QHK_DEBUG.exists() or LIB_QHK_DEBUG.stat().st_mtime < _newest(objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB_QHK_DEBUG), *map(str, objs)])
    return LIB_QHK_DEBUG


def build_host(force=False) -> Path | None:
    host_dir = CSRC / "host"
    sources = sorted(host_dir.glob("*.cpp")) if host_dir.exists() else []
    if not sources:
        return None
    BUILD.mkdir(exist_ok=True)
    jobs, objs = [], []
    for src in sources:
        obj = BUILD / ("host_" + src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append(["g++", *CXX_FLAGS, "-MD", "-MF", str(obj.with_suffix(".d")), "-c", str(src), "-o", str(obj)])
    _compile_many(jobs)
    if force or jobs or not LIB_HOST.exists() or LIB_HOST.stat().st_mtime < max(_newest(objs), LIB_QHK.stat().st_mtime):
        _run(["g++", "-shared", "-o", str(LIB_HOST), *map(str, objs), f"-L{PKG}", "-lqhk", "-Wl,-rpath,$ORIGIN"])
    return LIB_HOST


def build_bindings(force=False) -> Path | None:
    src = CSRC / "bindings.cpp"
    if not src.exists():
        return None
    import pybind11

    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = PKG / f"_core{suffix}"
    deps = [src, LIB_HOST, *(_headers())]
    if force or not out.exists() or out.stat().st_mtime < _newest(deps):
        _run(["g++", *CXX_FLAGS, "-shared", f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}",
              str(src), "-o", str(out), f"-L{PKG}", "-lqoraholo", "-lqhk", "-Wl,-rpath,$ORIGIN"])
    return out


def build(force=False, debug=False):
    build_qhk(force)
    build_host(force)
    build_bindings(force)
    if debug:
        build_qhk_debug(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, debug="--debug" in sys.argv)
    print("built", LIB_QHK, *([LIB_QHK_DEBUG] if "--debug" in sys.argv else []))
