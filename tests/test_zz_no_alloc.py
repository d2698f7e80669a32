"""The allocation-free unwrap entry point (qhk_unwrap_noalloc) through the C ABI, against the
planned entry point qhk_unwrap on the same inputs, on two calls in a row: the larger shape first,
then a smaller one, so that scratch left over from the first call would show in the second.
Callers that cannot allocate device memory -- a process whose memory is reserved by its own
allocator or budget, a real-time loop -- use it with buffers they own; its scratch is a static
device array shared by every call.

This file is collected last so that a failure here leaves every other test already run."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import host, rel_err

pytestmark = pytest.mark.gpu


def smooth_wrapped(count, ny, nx, seed):
    rng = np.random.default_rng(seed)
    z, y, x = np.indices((count, ny, nx)).astype(np.float32)
    phase = (25.0 * np.exp(-((x - nx * 0.45) ** 2 + (y - ny * 0.5) ** 2) / (0.05 * nx * ny))
             + (3.0 + z) * np.sin(x / nx * 3.0) + 0.04 * y + rng.normal(0, 0.1, (count, ny, nx)))
    return np.angle(np.exp(1j * phase.astype(np.float64))).astype(np.float32)


def test_unwrap_noalloc_matches_unwrap(cuda):
    import qoraholo_b200 as qh
    from qoraholo_b200 import capi

    for count, ny, nx, seed in ((2, 256, 256, 2), (3, 128, 96, 1)):
        w = smooth_wrapped(count, ny, nx, seed)
        expected = qh.unwrap(w)  # planned entry point (qhk_unwrap)
        d_in = cuda.from_numpy(w).cuda()
        d_out = cuda.full_like(d_in, float("nan"))
        capi.unwrap_noalloc(d_in.data_ptr(), d_out.data_ptr(), count, ny, nx)
        got = host(d_out)
        assert np.isfinite(got).all()
        assert rel_err(got, expected) < 1e-4
        # Same kernels and bit-identical tables: the two entry points agree bit for bit.
        assert np.array_equal(got, expected)


def test_unwrap_noalloc_rejects_oversized_requests(cuda):
    from qoraholo_b200 import capi

    d = cuda.zeros(4, dtype=cuda.float32, device="cuda")
    with pytest.raises(ValueError, match="at most"):
        capi.unwrap_noalloc(d.data_ptr(), d.data_ptr(), 1, 2048, 2048)
    with pytest.raises(ValueError, match="at most"):
        capi.unwrap_noalloc(d.data_ptr(), d.data_ptr(), 80, 512, 512)
