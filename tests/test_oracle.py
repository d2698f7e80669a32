"""The numpy oracle against the golden fixtures made by the reference itself (oracle/_ref built
from the reference sources; tests/golden/make_golden.py), and against oracle/_ref directly when
it is built. CPU only."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import contrast_err, golden, rel_err
from oracle import qh_oracle as O
from oracle import refimpl

GEOM = np.array([0.532, 1.337, 1.2, 0.2], np.float32)
CELL = np.array([[0.0, 0.4, -0.3, 2.5, 1.36], [0.0, 0.4, -0.3, 1.0, 1.38]], np.float32)


def test_dct_matches_reference_and_pocketfft():
    g = golden("dct")
    # Dct.MatchesPocketfftTypeTwo (tests/test_dct.cpp:22-37): 1e-4 abs against pocketfft x 0.5
    np.testing.assert_allclose(O.dct2(g["a"], 1), g["pocket_y"], atol=1e-4)
    np.testing.assert_allclose(O.dct2(g["a"], 2), g["pocket_x"], atol=1e-4)
    np.testing.assert_allclose(O.dct2(g["a"], 1), g["dct_y"], atol=1e-6)
    np.testing.assert_allclose(O.idct2(g["a"], 2), g["idct_x"], atol=1e-6)
    # Dct.InverseRoundTrips (tests/test_dct.cpp:39-47)
    for axis in (1, 2):
        np.testing.assert_allclose(O.idct2(O.dct2(g["a"], axis), axis), g["a"], atol=1e-5)


def test_field_extraction_matches_reference():
    for name in ("field", "field_negkx"):
        g = golden(name)
        out = O.extract_fields(g["holo"], tuple(g["center"]), float(g["radius"]), 0.0, int(g["out"]))
        assert rel_err(out, g["fields"]) < 1e-5


def test_sideband_matches_reference():
    g = golden("sideband")
    iy, ix, y, x, mag = O.find_sideband(g["holo"])
    assert (iy, ix) == (int(g["iy"]), int(g["ix"])) == (35, 35)
    assert abs(y - float(g["y"])) < 1e-4 and abs(x - float(g["x"])) < 1e-4
    # Field.FindsCarrierSideband (tests/test_field.cpp:39-50): 35.2 px within 0.05
    assert abs(y - 35.2) < 0.05 and abs(x - 35.2) < 0.05


def test_rytov_and_unwrap_match_reference():
    g = golden("rytov")
    assert rel_err(O.rytov(g["ratio"]), g["rytov"]) < 1e-5
    assert rel_err(O.unwrap(g["wrapped"]), g["unwrapped"]) < 1e-5


def test_reconstruct_matches_reference():
    g = golden("reconstruct")
    nm = float(g["geom"][1])
    cases = {"plain": {}, "gp_r2c": dict(iterations=5), "gp_c2c": dict(iterations=5, gp_transform="c2c"),
             "tv": dict(iterations=5, solver="tv"), "tv_nz34": dict(iterations=3, solver="tv", nz=34)}
    for name, kw in cases.items():
        ri, filled = O.reconstruct(g["fields"], g["illum"], g["geom"], **kw)
        assert contrast_err(ri, g[name], nm) < 1e-5, name
        assert filled == float(g[name + "_filled"]), name  # hit mask identical (EXPECT_DOUBLE_EQ)


def test_tv_prox_bitwise_against_reference():
    g = golden("tv_prox")
    p = [g["p0"][a].copy() for a in range(3)]
    x = O.tv_prox(g["b"], p, float(g["lam"]), int(g["inner"]))
    assert np.array_equal(x, g["x"])
    assert np.array_equal(np.stack(p), g["p"])


def test_bpm_matches_reference():
    g = golden("bpm")
    fwd = O.bpm_forward(g["ri"], g["illum"], GEOM)
    assert rel_err(fwd - 1, g["forward"] - 1) < 1e-5
    t = O.bpm_tables(24, 16, g["illum"], GEOM)
    xc = (g["ri"] - GEOM[1]).astype(np.float32)
    assert rel_err(O.bpm_vjp(xc, g["residual"], t), g["vjp"]) < 1e-5
    init = np.full((16, 24, 24), GEOM[1], np.float32)
    for batch in (0, 2):
        ri, loss = O.bpm_reconstruct(g["forward"], g["illum"], GEOM, init, iterations=3, batch=batch, tv_weight=1e-2)
        assert contrast_err(ri, g[f"rec_batch{batch}"], GEOM[1]) < 1e-4
        np.testing.assert_allclose(loss, g[f"loss_batch{batch}"], rtol=1e-5)


def test_phantom_generators_match_reference():
    g = golden("phantom")
    assert rel_err(O.forward_fields(CELL, g["illum"], GEOM, 32, "born") - 1, g["born"] - 1) < 1e-5
    assert rel_err(O.forward_fields(CELL, g["illum"], GEOM, 32, "rytov") - 1, g["rytov"] - 1) < 1e-5
    assert rel_err(O.forward_fields(CELL[:1], g["illum"], GEOM, 32, "exact") - 1, g["exact"] - 1) < 1e-5
    np.testing.assert_array_equal(O.render_phantom(CELL, GEOM, 12, 32), g["render"])
    np.testing.assert_allclose(O.synthesize_holograms(g["rytov"], g["illum"], GEOM, (1.0, 1.5)), g["holo"], rtol=1e-6)
    np.testing.assert_array_equal(O.circular_scan(49, 0.9, GEOM), g["scan49"])


def test_pipeline_chain_matches_reference_pipeline():
    g = golden("pipeline")
    c = tuple(g["center"])
    r = O.field_ratio(O.extract_fields(g["holo"], c, float(g["radius"]), 0, int(g["out"])),
                      O.extract_fields(g["bg"], c, float(g["radius"]), 0, int(g["out"])))
    ri, filled = O.reconstruct(O.rytov(r), g["illum"], g["geom"], iterations=5)
    assert contrast_err(ri, g["ri"], float(g["geom"][1])) < 1e-5
    assert filled == float(g["filled"])


def test_validation_errors():
    with pytest.raises(ValueError):
        O.unwrap(np.zeros((5, 6), np.float32))
    with pytest.raises(ValueError):
        O.reconstruct(np.zeros((2, 8, 8), np.complex64), np.zeros((3, 2), np.float32), GEOM)
    with pytest.raises(ValueError):
        O.crop_plan((10.0, 10.0), 64, radius=40.0, output_size=32)


@pytest.mark.skipif(not refimpl.available(), reason="oracle/_ref not built")
def test_oracle_against_reference_library_random_cases():
    rng = np.random.default_rng(11)
    il = refimpl.circular_scan(9, 0.9, GEOM)
    assert np.array_equal(il, O.circular_scan(9, 0.9, GEOM))
    fields = O.rytov(O.forward_fields(CELL, il, GEOM, 32, "rytov"))
    for kw in ({}, dict(iterations=2), dict(iterations=2, solver="tv", tv_inner=3)):
        a, fa = refimpl.reconstruct(fields, il, GEOM, **kw)
        b, fb = O.reconstruct(fields, il, GEOM, **kw)
        assert contrast_err(b, a, GEOM[1]) < 1e-5 and fa == fb
    b0 = rng.uniform(-0.1, 1, (6, 8, 12)).astype(np.float32)
    p0 = rng.uniform(-0.3, 0.3, (3, 6, 8, 12)).astype(np.float32)
    xr, pr = refimpl.tv_prox(b0, p0, 0.07, 5)
    p = [p0[a].copy() for a in range(3)]
    assert np.array_equal(O.tv_prox(b0, p, 0.07, 5), xr) and np.array_equal(np.stack(p), pr)


@pytest.mark.parametrize("n,nz,pixel", [(64, 64, 0.25), (256, 256, 0.11)])
def test_ewald_mapping_equals_the_reference_bitwise(n, nz, pixel):
    """The numpy mapping and Hermitian half data against the reference's own mapping (oracle/_ref's
    ref_ewald_half: its ewald_target, parity and hermitian_data), 49 views, up to the C2 size."""
    if not refimpl.available():
        pytest.skip("oracle/_ref not built")
    geom = np.array([0.532, 1.337, 1.2, pixel], np.float32)
    il = O.circular_scan(49, 0.9, geom)
    rng = np.random.default_rng(n)
    sp = (rng.standard_normal((49, n, n)) + 1j * rng.standard_normal((49, n, n))).astype(np.complex64)
    a_ref, hits_ref, filled_ref = refimpl.ewald_half(sp, il, geom, nz)
    pre, pim, w = O.ewald_map(sp, il, O.make_grid(n, nz, geom))
    f = w > 0
    pre = np.where(f, pre / np.where(f, w, 1), pre).astype(np.float32)
    pim = np.where(f, pim / np.where(f, w, 1), pim).astype(np.float32)
    a, hits = O.hermitian_half(pre, pim, w)
    assert np.array_equal(hits, hits_ref)
    assert np.array_equal(a, a_ref)
    assert int(np.count_nonzero(f)) == filled_ref
