"""Kernels with device bounds checks, run through the C ABI on seeded inputs (helper of
tests/test_debug_build.py, run as a script in a process of its own).

Usage: python tests/_debug_workload.py OUT.npz. The library is the one QHK_LIBRARY names (the
release build by default); capi.py is loaded on its own, without the package, so that the process
holds exactly one build of libqhk.so. Saves every result, the library's debug flag, its failed
checks and its wait timeouts.
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]


def load_capi():
    spec = importlib.util.spec_from_file_location("qhk_capi_standalone", ROOT / "qoraholo_b200" / "capi.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(out_path: str) -> None:
    capi = load_capi()
    rng = np.random.default_rng(20261204)
    dev = torch.device("cuda")
    out = {}

    # TV proximal step: the two-step FGP kernel (12 work volumes) and the one-step form (9).
    nz, ny, nx = 48, 64, 64
    b = torch.from_numpy(rng.standard_normal((nz, ny, nx)).astype(np.float32)).to(dev)
    for vols in (12, 9):
        x = torch.empty_like(b)
        work = torch.zeros((vols, nz, ny, nx), device=dev)
        capi.tv_prox_workspace(b.data_ptr(), x.data_ptr(), work.data_ptr(), vols, nz, ny, nx, 0.05, 10)
        out[f"tv_{vols}"] = x.cpu().numpy()

    # Uneven unwrap batch: register-engine sides (128, 256, 384, 512) and staged ones (192, 60 x 100).
    shapes = [(512, 512), (384, 384), (256, 256), (192, 192), (128, 128), (60, 100)]
    plan = capi.UnwrapBatch(shapes)
    images = [(rng.uniform(-np.pi, np.pi, s)).astype(np.float32) for s in shapes]
    d_in = torch.from_numpy(plan.pack(images)).to(dev)
    d_out = torch.empty_like(d_in)
    plan.run(d_in.data_ptr(), d_out.data_ptr())
    out["unwrap_batch"] = d_out.cpu().numpy()
    plan.close()

    # The allocation-free unwrap.
    w = torch.from_numpy(rng.uniform(-np.pi, np.pi, (2, 256, 256)).astype(np.float32)).to(dev)
    u = torch.empty_like(w)
    capi.unwrap_noalloc(w.data_ptr(), u.data_ptr(), 2, 256, 256)
    out["unwrap_noalloc"] = u.cpu().numpy()

    # Half-spectrum transforms on the register engine (axis and row passes).
    for shape in ((64, 64, 64), (32, 128, 256)):
        v = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(dev)
        half = torch.empty((shape[0], shape[1], shape[2] // 2 + 1), dtype=torch.complex64, device=dev)
        capi.rfft3(v.data_ptr(), half.data_ptr(), *shape)
        back = torch.empty_like(v)
        capi.irfft3(half.data_ptr(), back.data_ptr(), *shape, scale=1.0 / v.numel())
        out[f"rfft3_{shape}"] = half.cpu().numpy()
        out[f"irfft3_{shape}"] = back.cpu().numpy()

    # Reconstruction from fields: Ewald mapping of the half spectrum, k-space passes, FISTA-TV.
    count, n = 8, 64
    angles = 2 * np.pi * np.arange(count) / count
    illum = np.stack([0.4 * np.sin(angles), 0.4 * np.cos(angles)], 1).astype(np.float32)
    fields = (1 + 0.05 * (rng.standard_normal((count, n, n)) + 1j * rng.standard_normal((count, n, n))))
    geom = (0.532, 1.333, 1.2, 0.2)
    for solver in ("gp", "tv"):
        ri, filled = capi.reconstruct(fields.astype(np.complex64), illum, geom, iterations=3, solver=solver,
                                      tv_inner=4)
        out[f"reconstruct_{solver}"] = ri
        out[f"filled_{solver}"] = np.float64(filled)

    # BPM gradient (register-engine 2D transforms).
    xb = (0.01 * rng.standard_normal((16, 64, 64))).astype(np.float32)
    rb = (rng.standard_normal((4, 64, 64)) + 1j * rng.standard_normal((4, 64, 64))).astype(np.complex64)
    out["bpm_vjp"] = capi.bpm_vjp(xb, rb, illum[:4], geom)

    torch.cuda.synchronize()
    violations, where = capi.debug_violations()
    out["debug_enabled"] = np.int64(capi.debug_enabled())
    out["violations"] = np.int64(violations)
    out["where"] = np.array(where)
    out["wait_timeouts"] = np.int64(capi.wait_timeouts())
    np.savez(out_path, **out)


if __name__ == "__main__":
    main(sys.argv[1])
