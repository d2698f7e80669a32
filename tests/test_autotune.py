"""The launch-shape autotuner: plans built with it time their FFT axis tile widths and FGP tile
heights, record them, and reconstruct bitwise the same volume as plans with the default shapes."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import rel_err

pytestmark = pytest.mark.gpu

G = (0.532, 1.337, 1.2, 0.2)


def _run(torch, capi, n, nz, options):
    from oracle import qh_oracle as O

    il = O.circular_scan(9, 0.9, np.array(G, np.float32))
    rng = np.random.default_rng(4)
    fields = (rng.standard_normal((9, n, n)) + 1j * rng.standard_normal((9, n, n))).astype(np.complex64) * 0.05
    plan = capi.OdtPlan(n, 9, il, G, nz=nz, **options)
    d_f = torch.from_numpy(fields).cuda()
    out = torch.empty(plan.shape, dtype=torch.float32, device="cuda")
    plan.run(d_f.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.close()
    return out.cpu().numpy()


@pytest.mark.parametrize("n,nz,options", [
    (96, 64, dict(iterations=3, solver="tv", tv_inner=4)),
    (64, 48, dict(iterations=3, solver="gp")),
    (48, 32, dict(iterations=2, solver="gp", gp_transform="c2c")),
])
def test_tuned_and_default_shapes_give_the_same_volume(cuda, n, nz, options):
    from qoraholo_b200 import capi

    try:
        capi.autotune_enable(False)
        plain = _run(cuda, capi, n, nz, options)
        capi.autotune_enable(True)
        tuned = _run(cuda, capi, n, nz, options)
    finally:
        capi.autotune_enable(True)
    assert np.array_equal(plain, tuned)
    report = capi.autotune_report()
    assert "axis_cols" in report
    if options["solver"] == "tv":
        assert "fgp_rows" in report


@pytest.mark.parametrize("n,nz", [(64, 64), (128, 64), (64, 128)])
def test_every_axis_decomposition_matches_the_oracle(cuda, n, nz):
    """Each FFT decomposition of the axis passes (staged radix engine, register variants 1 and 2) gives
    the GP reconstruction within the oracle's tolerance, and variant 1 is the default's bits."""
    from oracle import qh_oracle as O
    from qoraholo_b200 import capi

    options = dict(iterations=3, solver="gp")
    il = O.circular_scan(9, 0.9, np.array(G, np.float32))
    rng = np.random.default_rng(4)
    fields = (rng.standard_normal((9, n, n)) + 1j * rng.standard_normal((9, n, n))).astype(np.complex64) * 0.05
    want, _ = O.reconstruct(fields, il, np.array(G, np.float32), nz=nz, **options)
    default = _run(cuda, capi, n, nz, options)
    try:
        for engine in (0, 1, 2):
            capi.fft_axis_engine(engine)
            got = _run(cuda, capi, n, nz, options)
            assert rel_err(got - G[1], want - G[1]) < 1e-4, engine
            if engine == 1:
                assert np.array_equal(got, default)
    finally:
        capi.fft_axis_engine(-1)


def test_radix_tuning_times_the_decompositions(cuda):
    from qoraholo_b200 import capi

    options = dict(iterations=2, solver="gp")
    try:
        capi.autotune_radix(True)
        tuned = _run(cuda, capi, 64, 80, options)
    finally:
        capi.autotune_radix(False)
    plain = _run(cuda, capi, 64, 80, options)
    assert "axis_engine" in capi.autotune_report()
    assert rel_err(tuned - G[1], plain - G[1]) < 1e-5
