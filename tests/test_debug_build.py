"""The debug build (QHK_DEBUG: device bounds checks in the tile loaders, work-queue items, line
indices and shared-memory layouts; `python qoraholo_b200/_build.py --debug`).

CPU: the release library reports the checks off and no failures, and both libraries export the
debug entry points. GPU: the same seeded workload (tests/_debug_workload.py) through the release and
the debug library, each in a process of its own: no check fails and no bounded wait runs out, and
every result of the debug build is bitwise the release build's -- the checks only observe.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
RELEASE = ROOT / "qoraholo_b200" / "libqhk.so"
DEBUG = ROOT / "qoraholo_b200" / "debug" / "libqhk.so"


def test_release_library_has_checks_off():
    lib = ctypes.CDLL(str(RELEASE))
    assert lib.qhk_debug_enabled() == 0
    n = ctypes.c_uint64(123)
    assert lib.qhk_debug_violations(ctypes.byref(n), 0) == 0
    assert n.value == 0


def test_debug_library_exports_the_abi():
    if not DEBUG.exists():
        pytest.skip("debug library not built (python qoraholo_b200/_build.py --debug)")
    out = subprocess.run(["nm", "-D", "--defined-only", str(DEBUG)], capture_output=True, text=True, check=True).stdout
    rel = subprocess.run(["nm", "-D", "--defined-only", str(RELEASE)], capture_output=True, text=True, check=True).stdout
    names = lambda s: {ln.split()[-1] for ln in s.splitlines() if " T qhk_" in ln}  # noqa: E731
    assert names(rel) and names(out) == names(rel)


def _run_workload(tmp_path, library, tag):
    env = dict(os.environ)
    if library is not None:
        env["QHK_LIBRARY"] = str(library)
    path = tmp_path / f"{tag}.npz"
    subprocess.run([sys.executable, str(ROOT / "tests" / "_debug_workload.py"), str(path)], env=env, check=True,
                   timeout=600)
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.gpu
def test_debug_build_finds_nothing_and_changes_nothing(tmp_path):
    assert DEBUG.exists(), "debug library missing: python qoraholo_b200/_build.py --debug"
    rel = _run_workload(tmp_path, None, "release")
    dbg = _run_workload(tmp_path, DEBUG, "debug")
    assert int(rel["debug_enabled"]) == 0 and int(dbg["debug_enabled"]) == 1
    assert int(dbg["violations"]) == 0, str(dbg["where"])
    assert int(rel["wait_timeouts"]) == 0 and int(dbg["wait_timeouts"]) == 0
    skip = {"debug_enabled", "violations", "where", "wait_timeouts"}
    assert set(rel) == set(dbg)
    for k in sorted(set(rel) - skip):
        assert rel[k].dtype == dbg[k].dtype and rel[k].shape == dbg[k].shape, k
        assert rel[k].tobytes() == dbg[k].tobytes(), f"{k}: the debug build changed the result"
