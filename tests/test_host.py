"""Host-side checks that need no GPU: the C ABI library loads and exports every function the
header declares; the Python package imports and validates arguments before touching a device;
the benchmark's workload and rank aggregation."""

from __future__ import annotations

import ctypes
import math
import os
import re
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include" / "qoraholo_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qhk_[a-z0-9_]+)\s*\(", text)))


def test_c_abi_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ROOT / "qoraholo_b200" / "libqhk.so"))
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_c_abi_reports_errors_without_a_device():
    from qoraholo_b200 import capi

    lib = capi.lib()
    assert lib.qhk_last_error() is not None
    g = capi.Geometry(0.532, 1.337, 1.2, 0.2)
    o = capi.odt_options(iterations=1)
    h = ctypes.c_void_p()
    il = np.zeros((3, 2), np.float32)
    # odd side: invalid argument before any device work
    code = lib.qhk_odt_create(ctypes.byref(h), 7, 3, capi.host_ptr(il), ctypes.byref(g), ctypes.byref(o))
    assert code == capi.INVALID_ARGUMENT
    assert "even" in lib.qhk_last_error().decode()


def test_python_api_validates_before_device():
    import qoraholo_b200 as qh

    g = qh.Geometry(wavelength=0.532, n_medium=1.337, na=1.2, pixel=0.2)
    with pytest.raises(ValueError):
        qh.unwrap(np.zeros((5, 6), np.float32))
    with pytest.raises(ValueError):
        qh.extract_fields(np.zeros((1, 8, 10), np.float32), center=(2, 2))
    with pytest.raises(ValueError):
        qh.reconstruct(np.zeros((2, 8, 8), np.complex64), np.zeros((3, 2), np.float32), g)
    with pytest.raises(ValueError):
        qh.circular_scan(0, 0.9, g)
    with pytest.raises(RuntimeError):
        qh.reconstruct(np.zeros((3, 8, 8), np.complex64), np.zeros((3, 2), np.float32), g, backend="cpu")
    with pytest.raises(ValueError):
        qh.Pipeline(3, 32, (8, 8), np.zeros((3, 2), np.float32), g, upload_chunks=0)


def test_circular_scan_matches_oracle():
    import qoraholo_b200 as qh
    from oracle import qh_oracle as O

    g = qh.Geometry(wavelength=0.532, n_medium=1.337, na=1.2, pixel=0.2)
    assert np.array_equal(qh.circular_scan(49, 0.9, g), O.circular_scan(49, 0.9, (0.532, 1.337, 1.2, 0.2)))


def test_bench_cell_is_nested():
    import bench

    # every shape lies entirely inside or outside each earlier one (painter's order stays analytic)
    rng = np.random.default_rng(0)
    for i, (_, c, a, _) in enumerate(bench.CELL):
        u = rng.normal(size=(4000, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        pts = np.asarray(c) + u * np.asarray(a)
        for earlier in bench.CELL[:i]:
            inside = [bench._inside(earlier, *p) for p in pts]
            assert all(inside) or not any(inside)


def test_bench_percentile_and_single_rank_rate():
    import bench

    assert bench.percentile([1.0, 2.0, 3.0, 4.0], 0.5) == 2.0
    assert bench.percentile(list(range(1, 101)), 0.99) == 99
    max_ms, value = bench.combine_ranks(2000.0, 10, 1)
    assert max_ms == 2000.0 and math.isclose(value, 5.0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = 1000.0 * (rank + 1)  # rank 1 is slower
    out[rank] = bench.combine_ranks(local, 4, world, dist, "cpu")
    dist.destroy_process_group()


def test_bench_combines_ranks_with_gloo():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        results = dict(out)
    for rank in range(world):
        max_ms, value = results[rank]
        assert max_ms == 2000.0  # max over ranks
        assert math.isclose(value, world * 4 * 1000.0 / 2000.0)
