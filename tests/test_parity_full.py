"""Parity at the full sizes of the benchmark configurations, against the reference's own CPU build
(oracle/_ref: its src/ and src/cpu/ sources compiled unmodified) on the same inputs. The bar is the
reference's own CUDA-against-CPU bar (tests/test_cuda.cpp:74-115): index-contrast error <= 1e-4 and
the filled fraction exactly equal; the Ewald mapping's data and hit counts bit for bit; the BPM
gradient <= 1e-4 (tests/test_cuda.cpp:140-160). Inputs are seeded synthetic phantoms with each
configuration's shapes, made with bench.py's numpy fixture generators (no reference code):

  C1  49 x 256^2 holograms -> 128^2 fields -> 128^3 Gerchberg-Papoulis, 20 iterations (bead)
  C2  49 x 512^2 -> 256^2 -> 256^3 FISTA-TV 20 x 10, TV weight 1e-2 (synthetic cell)
  C3  97 x 1024^2 -> 384^2 -> 384^3 Gerchberg-Papoulis, 20 iterations (cell), the serving mix's
      largest request
  C5  BPM gradient, 256^2 x 128 slices, all 49 views (20 overlapping spheres)
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import bench
from conftest import contrast_err, dev, host
from oracle import qh_oracle as O
from oracle import refimpl

pytestmark = [pytest.mark.gpu, pytest.mark.slow,
              pytest.mark.skipif(not refimpl.available(), reason="oracle/_ref (the reference CPU build) is missing")]

NM = bench.N_MEDIUM


def _geom(pixel):
    return (bench.WAVELENGTH, NM, bench.NA, pixel)


def _stacks(shapes, count, n, holo_pixel, carrier, device=None):
    illum = bench.circular_scan(count, 0.9)
    ratio = bench.phantom_fields(shapes, illum, n, holo_pixel, device)
    holo = bench.holograms(ratio, illum, holo_pixel, carrier, seed=1)
    bg = bench.holograms(np.ones_like(ratio), illum, holo_pixel, carrier, seed=2)
    return illum, holo, bg


def _ours(count, n, carrier, illum, field_pixel, holo, bg, **kw):
    import qoraholo_b200 as qh

    g = qh.Geometry(wavelength=bench.WAVELENGTH, n_medium=NM, na=bench.NA, pixel=field_pixel)
    p = qh.Pipeline(count, n, (carrier, carrier), illum, g, **kw)
    p.set_background(bg)
    ri = np.array(p.run(holo))
    return ri, p.filled


def _reference(holo, bg, carrier, radius, out, illum, field_pixel, **kw):
    ri, filled, _ = refimpl.pipeline(holo, bg, (carrier, carrier), radius, out, illum, _geom(field_pixel), **kw)
    return ri, filled


def test_c1_bead_128cubed_gp20_matches_reference_cpu(cuda):
    bead = [("ellipsoid", (0.0, 0.0, 0.0), (2.5, 2.5, 2.5), 1.360)]
    illum, holo, bg = _stacks(bead, 49, 256, 0.1, 70)
    kw = dict(iterations=20, solver="gp")
    ri, filled = _ours(49, 256, 70, illum, 0.2, holo, bg, radius=59.0, output_size=128, **kw)
    ref, ref_filled = _reference(holo, bg, 70, 59.0, 128, illum, 0.2, **kw)
    assert ri.shape == (128, 128, 128)
    assert contrast_err(ri, ref, NM) <= 1e-4
    assert filled == ref_filled


def test_c2_cell_256cubed_fista_tv_20x10_matches_reference_cpu(cuda):
    illum, holo, bg = bench.make_inputs()
    kw = dict(iterations=bench.ITERATIONS, solver="tv", tv_weight=bench.TV_WEIGHT, tv_inner=bench.TV_INNER)
    ri, filled = _ours(bench.COUNT, bench.HOLO_N, bench.CARRIER_PX, illum, bench.FIELD_PIXEL, holo, bg,
                       radius=bench.RADIUS, output_size=bench.FIELD_N, **kw)
    ref, ref_filled = _reference(holo, bg, bench.CARRIER_PX, bench.RADIUS, bench.FIELD_N, illum, bench.FIELD_PIXEL,
                                 **kw)
    assert contrast_err(ri, ref, NM) <= 1e-4
    assert filled == ref_filled


def test_c3_cell_384cubed_gp20_matches_reference_cpu(cuda):
    n, out, hpix, carrier, radius = 1024, 384, 0.04125, 212, 98.0
    illum, holo, bg = _stacks(bench.CELL, 97, n, hpix, carrier, device="cuda")
    kw = dict(iterations=20, solver="gp")
    ri, filled = _ours(97, n, carrier, illum, hpix * n / out, holo, bg, radius=radius, output_size=out, **kw)
    ref, ref_filled = _reference(holo, bg, carrier, radius, out, illum, hpix * n / out, **kw)
    assert contrast_err(ri, ref, NM) <= 1e-4
    assert filled == ref_filled


@pytest.mark.parametrize("n,count,pixel", [(256, 49, 0.11), (384, 97, 0.11)])
def test_ewald_mapping_bitwise_against_the_reference_at_full_size(cuda, n, count, pixel):
    """k_map_half's half-spectrum data, hit counts and filled count against the reference's own
    mapping (ref_ewald_half) on the spectra of real Rytov fields of the C2 / C3 geometry."""
    from qoraholo_b200 import capi

    geom = np.array(_geom(pixel), np.float32)
    illum = bench.circular_scan(count, 0.9)
    ratio = bench.phantom_fields(bench.CELL, illum, n, pixel, "cuda")
    spectra = np.fft.fft2(O.rytov(ratio)).astype(np.complex64)
    a_ref, hits_ref, filled_ref = refimpl.ewald_half(spectra, illum, geom, n)
    h = n // 2 + 1
    a = cuda.zeros((n, n, h), dtype=cuda.complex64, device="cuda")
    hits = cuda.zeros((n, n, h), dtype=cuda.uint8, device="cuda")
    cnt = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    ts = dev(cuda, spectra)
    capi.ewald_map(ts.data_ptr(), count, n, n, illum, geom, 1, a.data_ptr(), hits.data_ptr(), cnt.data_ptr())
    assert np.array_equal(host(hits), hits_ref)
    assert np.array_equal(host(a), a_ref)
    assert int(host(cnt)[0]) == filled_ref


def test_c5_bpm_gradient_all_49_views_matches_reference_vjp(cuda):
    """The hand-written adjoint behind torch.autograd (checkpoint every 16 slices) against the
    reference's bpm_vjp over all 49 views, at the C5 size, from the homogeneous starting point."""
    import torch

    from qoraholo_b200.autograd import BpmModel

    nz, n, pixel = bench.BPM_NZ, bench.BPM_N, bench.BPM_PIXEL
    geom = _geom(pixel)
    rng = np.random.default_rng(17)
    spheres = np.array([[rng.uniform(-5, 5), rng.uniform(-8, 8), rng.uniform(-8, 8), rng.uniform(1, 3),
                         NM + rng.uniform(0.005, 0.05)] for _ in range(20)], np.float32)
    truth = O.render_phantom(spheres, geom, nz, n)
    illum = bench.circular_scan(bench.BPM_VIEWS, 0.9)
    x0 = np.full((nz, n, n), NM, np.float32)
    data = refimpl.bpm_forward(truth, illum, geom)
    r = (refimpl.bpm_forward(x0, illum, geom) - data).astype(np.complex64)
    want = refimpl.bpm_vjp(x0 - NM, r, illum, geom)

    import qoraholo_b200 as qh

    g = qh.Geometry(wavelength=bench.WAVELENGTH, n_medium=NM, na=bench.NA, pixel=pixel)
    model = BpmModel(nz, n, illum, g, checkpoint_every=bench.BPM_EVERY)
    x = torch.from_numpy(x0).cuda().requires_grad_(True)
    model(x).backward(torch.from_numpy(r).cuda())
    got = x.grad.cpu().numpy()
    model.plan.close()
    err = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    assert err <= 1e-4, err
    assert math.isfinite(err)
