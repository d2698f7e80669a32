"""Bounded device waits become error statuses. The two-step FGP kernel waits for its TMA box loads
on mbarriers with an iteration limit; a wait that runs out is counted in the calling plan's own
device counter, the kernel leaves after a bounded wait for each load it still has in flight, and
the call that synchronises on the work returns QHK_TIMEOUT (a RuntimeError here). A correct run
never runs out, so the timeout path is exercised with the pipeline's probe: one bounded wait, in
the same form, on an mbarrier that nothing arrives at -- no load in flight, nothing that faults or
hangs -- after which the pipeline must still give bitwise its earlier result."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = np.array([0.532, 1.337, 1.2, 0.2], np.float32)


def _inputs(count=9, n=64, out=32):
    from oracle import qh_oracle as O

    hg = G.copy()
    hg[3] = G[3] * out / n
    il = O.circular_scan(count, 0.9, G)
    c = 18 / (n * hg[3])
    sph = np.array([[0.0, 0.3, -0.2, 1.5, G[1] + 0.02]], np.float32)
    holo = O.synthesize_holograms(O.forward_fields(sph, il, hg, n), il, hg, carrier=(c, c), noise=0.02, seed=1)
    bg = O.synthesize_holograms(np.ones((count, n, n), np.complex64), il, hg, carrier=(c, c), noise=0.02, seed=2)
    return il, holo.astype(np.float32), bg.astype(np.float32)


def test_wait_that_runs_out_is_reported_and_the_pipeline_stays_usable(cuda):
    from qoraholo_b200 import capi

    il, holo, bg = _inputs()
    # 32^3 FISTA-TV with an even inner count: the two-step (TMA) FGP kernel runs.
    p = capi.Pipeline(9, 64, (18, 18), il, tuple(float(v) for v in G), radius=14.0, output_size=32, iterations=3,
                      solver="tv", tv_inner=4)
    p.set_background(bg)
    p.input[...] = holo
    p.process()
    before = p.output.copy()
    p.check_waits()  # nothing ran out

    with pytest.raises(capi.QhkError, match="bounded device wait ran out") as err:
        p.wait_probe(polls=2000)
    assert err.value.code == capi.TIMEOUT

    # Reported once: the next check is clean, and the pipeline computes the same volume again.
    p.check_waits()
    p.input[...] = holo
    p.process()
    assert np.array_equal(p.output, before)
    n = cuda.empty(0)  # the context still takes new work
    assert n.numel() == 0
    p.close()


def test_wait_probe_rejects_unbounded_limits(cuda):
    from qoraholo_b200 import capi

    il, _, bg = _inputs()
    p = capi.Pipeline(9, 64, (18, 18), il, tuple(float(v) for v in G), radius=14.0, output_size=32, iterations=1,
                      solver="gp")
    for polls in (0, -1, (1 << 20) + 1):
        with pytest.raises(ValueError, match="polls"):
            p.wait_probe(polls)
    p.close()
