"""Uneven batches in single launches: the unwrap of images of mixed sizes packed in one buffer
(persistent kernels draining an (image, tile) queue) gives for every image bitwise what the
per-size unwrap gives, directly and replayed as a CUDA graph, and agrees with the oracle."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def phase_map(rng, ny, nx):
    """A wrapped phase map: 3-6 Gaussians plus a tilt, peak-to-peak ~U[10, 60] rad, plus N(0, 0.1)."""
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    surf = rng.uniform(-1, 1) * y / ny + rng.uniform(-1, 1) * x / nx
    for _ in range(rng.integers(3, 7)):
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        sy, sx = rng.uniform(0.05, 0.3) * ny, rng.uniform(0.05, 0.3) * nx
        surf += rng.uniform(-1, 1) * np.exp(-((y - cy) / sy) ** 2 - ((x - cx) / sx) ** 2)
    surf = (surf - surf.min()) / max(np.ptp(surf), 1e-9) * rng.uniform(10, 60)
    surf += rng.normal(0, 0.1, surf.shape)
    return np.angle(np.exp(1j * surf)).astype(np.float32)


@pytest.fixture(scope="module")
def batch(cuda):
    rng = np.random.default_rng(12)
    sides = [128, 192, 256, 384, 512]
    shapes = [(int(s), int(s)) for s in rng.choice(sides, 24)] + [(96, 160), (160, 96), (64, 64), (2, 4)]
    images = [phase_map(rng, ny, nx) for ny, nx in shapes]
    return shapes, images


def test_uneven_batch_equals_per_image_unwrap(cuda, batch):
    import qoraholo_b200 as qh
    from qoraholo_b200 import capi

    shapes, images = batch
    plan = capi.UnwrapBatch(shapes)
    d_in = cuda.from_numpy(plan.pack(images)).cuda()
    outs = []
    d_out = cuda.zeros(plan.total, dtype=cuda.float32, device="cuda")
    for graph in (False, True, True):  # direct, then captured, then replayed
        d_out.zero_()
        plan.run(d_in.data_ptr(), d_out.data_ptr(), 0, graph=graph)
        cuda.cuda.synchronize()
        outs.append(d_out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    for img, got in zip(images, plan.unpack(outs[0])):
        assert np.array_equal(got, qh.unwrap(img)), img.shape
    plan.close()


def test_uneven_batch_on_unaligned_buffers(cuda, batch):
    """Buffers that start 4 bytes past a 16-byte boundary (e.g. tensor views) give the same bits."""
    from qoraholo_b200 import capi

    shapes, images = batch
    plan = capi.UnwrapBatch(shapes)
    packed = cuda.from_numpy(plan.pack(images))
    d_in = cuda.zeros(plan.total + 1, dtype=cuda.float32, device="cuda")
    d_in[1:] = packed.cuda()
    d_out = cuda.zeros(plan.total + 1, dtype=cuda.float32, device="cuda")
    plan.run(d_in[1:].data_ptr(), d_out[1:].data_ptr())
    ref_in = packed.cuda()
    ref_out = cuda.zeros(plan.total, dtype=cuda.float32, device="cuda")
    plan.run(ref_in.data_ptr(), ref_out.data_ptr())
    cuda.cuda.synchronize()
    assert np.array_equal(d_out[1:].cpu().numpy(), ref_out.cpu().numpy())
    plan.close()


def test_uneven_batch_matches_the_oracle(cuda, batch):
    from oracle import qh_oracle as O
    from qoraholo_b200 import capi

    shapes, images = batch
    pick = [0, 5, len(images) - 4, len(images) - 3]
    sub = [images[i] for i in pick]
    plan = capi.UnwrapBatch([shapes[i] for i in pick])
    d_in = cuda.from_numpy(plan.pack(sub)).cuda()
    d_out = cuda.empty(plan.total, dtype=cuda.float32, device="cuda")
    plan.run(d_in.data_ptr(), d_out.data_ptr())
    cuda.cuda.synchronize()
    for img, got in zip(sub, plan.unpack(d_out.cpu().numpy())):
        want = O.unwrap(img[None])[0]
        assert rel_err(got, want) < 1e-4


def test_uneven_batch_rejects_odd_sizes(cuda):
    from qoraholo_b200 import capi

    with pytest.raises(ValueError):
        capi.UnwrapBatch([(64, 64), (63, 64)])


# ---- batches of same-geometry reconstructions -------------------------------------------------

G = np.array([0.532, 1.337, 1.2, 0.2], np.float32)


def _stacks(B, count=9, n=64, out=32, seed=3):
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


@pytest.mark.parametrize("odt", [dict(iterations=4, solver="gp"), dict(iterations=0),
                                 dict(iterations=3, solver="gp", gp_transform="c2c", nz=24),
                                 dict(iterations=3, solver="tv", tv_weight=1e-2, tv_inner=4),
                                 dict(iterations=2, solver="tv", tv_inner=3, nz=40)])
def test_batched_pipeline_equals_single_requests(cuda, odt):
    from qoraholo_b200 import capi

    B = 5
    il, bg, stacks = _stacks(B)
    geom = tuple(float(v) for v in G)
    kw = dict(radius=14.0, output_size=32, **odt)
    single = capi.Pipeline(9, 64, (18, 18), il, geom, **kw)
    single.set_background(bg)
    want = []
    for h in stacks:
        single.input[...] = h
        single.process()
        want.append(single.output.copy())
    batched = capi.Pipeline(9, 64, (18, 18), il, geom, batch=B, **kw)
    batched.set_background(bg)
    d_holo = cuda.from_numpy(np.concatenate(stacks)).cuda()
    d_index = cuda.empty(batched.shape, dtype=cuda.float32, device="cuda")
    for run in (batched.process_device, batched.process_device_graph, batched.process_device_graph,
                batched.process_device_graph):
        d_index.zero_()
        run(d_holo.data_ptr(), d_index.data_ptr())
        got = d_index.cpu().numpy()
        for b in range(B):
            assert np.array_equal(got[b], want[b]), b
    assert np.all(batched.filled_batch() == single.result()[0])
    batched.input[...] = np.concatenate(stacks)
    batched.process()
    assert np.array_equal(batched.output, np.stack(want))


