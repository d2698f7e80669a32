"""Pipeline runs on caller host memory (qhk_pipeline_run, qoraholo.Pipeline.run): the holograms are
staged by the host copy threads chunk by chunk and the volume copied out part by part, and the
volume is bitwise the one process() leaves in the pipeline's own page-locked output -- for any
number of upload chunks, batched pipelines, caller buffers that are not page aligned, page-locked
caller buffers (transferred directly), and the pipeline's own buffers passed as source and
destination."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = np.array([0.532, 1.337, 1.2, 0.2], np.float32)


def _stacks(B, count=9, n=64, out=34, seed=5):
    from oracle import qh_oracle as O

    rng = np.random.default_rng(seed)
    hg = G.copy()
    hg[3] = G[3] * out / n
    il = O.circular_scan(count, 0.9, G)
    c = 18 / (n * hg[3])
    bg = O.synthesize_holograms(np.ones((count, n, n), np.complex64), il, hg, carrier=(c, c), noise=0.02, seed=99)
    stacks = []
    for b in range(B):
        sph = np.array([[0.0, rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(1.0, 2.0),
                         G[1] + rng.uniform(0.01, 0.04)]], np.float32)
        ratio = O.forward_fields(sph, il, hg, n)
        stacks.append(O.synthesize_holograms(ratio, il, hg, carrier=(c, c), noise=0.02, seed=b + 1).astype(np.float32))
    return il, bg.astype(np.float32), stacks


def _pipeline(capi, il, bg, **kw):
    p = capi.Pipeline(9, 64, (18, 18), il, tuple(float(v) for v in G), radius=14.0, output_size=34, **kw)
    p.set_background(bg)
    return p


def _processed(p, holo):
    p.input[...] = holo
    p.process()
    return p.output.copy(), p.result()[0]


@pytest.mark.parametrize("odt", [dict(iterations=3, solver="tv", tv_inner=4, nz=26),
                                 dict(iterations=4, solver="gp")])
@pytest.mark.parametrize("chunks", [1, 4, 9])
def test_run_on_host_memory_equals_process(cuda, odt, chunks):
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(2)
    p = _pipeline(capi, il, bg, upload_chunks=chunks, **odt)
    for holo in stacks:
        want, filled = _processed(p, holo)
        got = p.run(holo)
        assert got is not p.output and np.array_equal(got, want)
        assert p.result()[0] == filled
        # a destination that is not page aligned (4 bytes past an aligned start), given by the caller
        raw = np.empty(got.size + 1, np.float32)
        dst = raw[1:].reshape(got.shape)
        assert dst.ctypes.data % 4096 != 0
        assert p.run(holo, out=dst) is dst and np.array_equal(dst, want)
    p.close()


def test_run_with_the_pipelines_own_buffers(cuda):
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(1)
    p = _pipeline(capi, il, bg, iterations=2, solver="gp", upload_chunks=3)
    want, _ = _processed(p, stacks[0])
    p.output[...] = 0
    assert p.run(p.input, out=p.output) is p.output  # source and destination are the staging buffers
    assert np.array_equal(p.output, want)
    p.close()


def test_batched_run_equals_batched_process(cuda):
    from qoraholo_b200 import capi

    B = 3
    il, bg, stacks = _stacks(B)
    p = _pipeline(capi, il, bg, iterations=3, solver="gp", batch=B)
    holo = np.concatenate(stacks)
    want, _ = _processed(p, holo)
    got = p.run(holo)
    assert got.shape == (B,) + p.shape[1:] and np.array_equal(got, want)
    p.close()


def test_run_rejects_wrong_shapes(cuda):
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(1)
    p = _pipeline(capi, il, bg, iterations=1, solver="gp")
    with pytest.raises(ValueError):
        p.run(stacks[0][:8])
    with pytest.raises(ValueError):
        p.run(stacks[0], out=np.empty((3, 3), np.float32))
    p.close()


def test_public_pipeline_run_equals_process(cuda):
    """qoraholo_b200.Pipeline.run (numpy in, new numpy out) through qhk_pipeline_run equals the
    C ABI's input -> process -> output on the same holograms."""
    import qoraholo_b200 as qh
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(2)
    geom = qh.Geometry(wavelength=float(G[0]), n_medium=float(G[1]), na=float(G[2]), pixel=float(G[3]))
    kw = dict(iterations=3, solver="tv", tv_inner=4)
    api = qh.Pipeline(9, 64, (18, 18), il, geom, radius=14.0, output_size=34, upload_chunks=4, **kw)
    api.set_background(bg)
    ref = _pipeline(capi, il, bg, upload_chunks=4, **kw)
    for holo in stacks:
        want, filled = _processed(ref, holo)
        got = api.run(holo)
        assert got.dtype == np.float32 and got.shape == ref.shape
        assert np.array_equal(got, want) and api.filled == filled
        assert api.timings["total"] > 0
    ref.close()


def test_run_on_page_locked_buffers_equals_process(cuda):
    """Page-locked holograms and volume (qhk_pinned_alloc) are transferred directly."""
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(2)
    p = _pipeline(capi, il, bg, iterations=3, solver="tv", tv_inner=4, upload_chunks=4)
    holo = capi.pinned_array(stacks[0].shape)
    out = capi.pinned_array(p.shape)
    for h in stacks:
        want, _ = _processed(p, h)
        holo[...] = h
        out[...] = -1.0
        assert p.run(holo, out=out) is out and np.array_equal(out, want)
    p.close()


def test_public_results_stay_valid_across_runs(cuda):
    """Pipeline.run returns arrays in recycled page-locked buffers: a result that is still held is
    never written by later runs, and released ones are reused."""
    import qoraholo_b200 as qh
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(3)
    geom = qh.Geometry(wavelength=float(G[0]), n_medium=float(G[1]), na=float(G[2]), pixel=float(G[3]))
    api = qh.Pipeline(9, 64, (18, 18), il, geom, radius=14.0, output_size=34, iterations=2)
    api.set_background(bg)
    held = [api.run(h) for h in stacks]  # three live results
    copies = [r.copy() for r in held]
    for _ in range(3):
        api.run(stacks[0])  # released at once, its buffer reused by the next run
    for r, c in zip(held, copies):
        assert np.array_equal(r, c)
    assert not np.array_equal(held[0], held[1])


@pytest.mark.parametrize("odt", [dict(iterations=3, solver="tv", tv_inner=4, nz=26),
                                 dict(iterations=4, solver="gp")])
@pytest.mark.parametrize("items,chunks", [(1, 1), (2, 4), (5, 3)])
def test_stream_equals_runs(cuda, odt, items, chunks):
    """qhk_pipeline_run_stream over `items` different stacks gives, volume by volume, bitwise what
    qhk_pipeline_run gives for each stack (the two device volumes alternate, the transfers overlap
    the solves), into a new array or a caller array that is not page aligned; filled is the last
    stack's; a single run afterwards is unaffected. From a volume slot's second use on, its solve is
    replayed as a CUDA graph (captured on the third stack, or in the second call), so items = 5 and
    the second call cover capture and replay."""
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(items, seed=11)
    p = _pipeline(capi, il, bg, upload_chunks=chunks, **odt)
    want, filled = [], []
    for h in stacks:
        want.append(p.run(h))
        filled.append(p.result()[0])
    holo = np.stack(stacks)
    got = p.run_stream(holo)
    assert got.shape == (items,) + tuple(p.shape)
    for i in range(items):
        assert np.array_equal(got[i], want[i]), i
    assert p.result()[0] == filled[-1] and p.result()[1]["total"] > 0
    raw = np.empty(got.size + 1, np.float32)
    dst = raw[1:].reshape(got.shape)
    assert p.run_stream(holo, out=dst) is dst and np.array_equal(dst, got)
    assert np.array_equal(p.run(stacks[0]), want[0])
    p.close()


def test_stream_on_page_locked_buffers(cuda):
    """Page-locked holograms and volumes go straight between the caller's buffers and the device."""
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(3, seed=12)
    p = _pipeline(capi, il, bg, iterations=3, solver="tv", tv_inner=4, upload_chunks=4)
    want = [p.run(h) for h in stacks]
    holo = capi.pinned_array((3,) + stacks[0].shape)
    out = capi.pinned_array((3,) + tuple(p.shape))
    holo[...] = np.stack(stacks)
    out[...] = -1.0
    assert p.run_stream(holo, out=out) is out
    for i in range(3):
        assert np.array_equal(out[i], want[i]), i
    p.close()


def test_batched_stream_equals_batched_runs(cuda):
    from qoraholo_b200 import capi

    B, items = 2, 3
    il, bg, stacks = _stacks(B * items, seed=13)
    p = _pipeline(capi, il, bg, iterations=3, solver="gp", batch=B)
    inputs = [np.concatenate(stacks[B * i:B * (i + 1)]) for i in range(items)]
    want = [p.run(h) for h in inputs]
    got = p.run_stream(np.stack(inputs))
    assert got.shape == (items, B) + tuple(p.shape[1:])
    for i in range(items):
        assert np.array_equal(got[i], want[i]), i
    p.close()


def test_public_pipeline_run_stream(cuda):
    """qoraholo_b200.Pipeline.run_stream ((items, count, N, N) numpy in, (items, nz, n, n) out) equals
    Pipeline.run per stack, and rejects inputs of the wrong shape."""
    import qoraholo_b200 as qh

    il, bg, stacks = _stacks(3, seed=14)
    geom = qh.Geometry(wavelength=float(G[0]), n_medium=float(G[1]), na=float(G[2]), pixel=float(G[3]))
    api = qh.Pipeline(9, 64, (18, 18), il, geom, radius=14.0, output_size=34, upload_chunks=3, iterations=3,
                      solver="tv", tv_inner=4)
    api.set_background(bg)
    want = [api.run(h).copy() for h in stacks]
    got = api.run_stream(np.stack(stacks))
    assert got.shape == (3,) + want[0].shape
    for i in range(3):
        assert np.array_equal(got[i], want[i]), i
    with pytest.raises(ValueError):
        api.run_stream(stacks[0])
    with pytest.raises(ValueError):
        api.run_stream(np.stack(stacks)[:, :8])


def test_stream_rejects_wrong_shapes(cuda):
    from qoraholo_b200 import capi

    il, bg, stacks = _stacks(1)
    p = _pipeline(capi, il, bg, iterations=1, solver="gp")
    with pytest.raises(ValueError):
        p.run_stream(stacks[0])
    with pytest.raises(ValueError):
        p.run_stream(stacks[0][None], out=np.empty((1, 3, 3), np.float32))
    p.close()
