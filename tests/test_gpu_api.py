"""The public Python API (qoraholo_b200, the reference's function signatures) on the device,
against the reference's golden fixtures, the oracle, and the known answers of the reference's
own tests (tests/test_field.cpp, test_unwrap.cpp, test_odt.cpp, test_cuda.cpp, test_pipeline.cpp,
test_bpm.cpp, python/tests/test_qoraholo.py)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import contrast_err, golden, rel_err
from oracle import qh_oracle as O

pytestmark = pytest.mark.gpu

G = np.array([0.532, 1.337, 1.2, 0.2], np.float32)
CELL = np.array([[0.0, 0.4, -0.3, 2.5, 1.36], [0.0, 0.4, -0.3, 1.0, 1.38]], np.float32)


@pytest.fixture(scope="module")
def qh(cuda):
    import qoraholo_b200

    assert qoraholo_b200.cuda_available()
    return qoraholo_b200


def geom(qh, g):
    return qh.Geometry(wavelength=float(g[0]), n_medium=float(g[1]), na=float(g[2]), pixel=float(g[3]))


def spheres(qh, s):
    return [qh.Sphere(z=float(a), y=float(b), x=float(c), radius=float(r), n=float(n)) for a, b, c, r, n in s]


# ---- field retrieval ---------------------------------------------------------------------------


@pytest.mark.parametrize("name", ["field", "field_negkx"])
def test_extract_fields_matches_reference(qh, name):
    # Cuda.FieldExtractionMatchesCpu / AcrossZeroKx (tests/test_cuda.cpp:37-66): 1e-4 relative
    g = golden(name)
    out = qh.extract_fields(g["holo"], center=tuple(g["center"]), radius=float(g["radius"]), output_size=int(g["out"]))
    assert rel_err(out, g["fields"]) < 1e-4


def test_find_sideband_matches_reference(qh):
    # Field.FindsCarrierSideband (tests/test_field.cpp:39-50)
    g = golden("sideband")
    s = qh.find_sideband(g["holo"][0])
    assert (s.iy, s.ix) == (35, 35)
    assert abs(s.y - float(g["y"])) < 1e-3 and abs(s.x - float(g["x"])) < 1e-3
    assert abs(s.y - 35.2) < 0.05 and abs(s.x - 35.2) < 0.05


def test_synthetic_hologram_gives_forward_field(qh):
    # Field.SyntheticHologramGivesForwardField (tests/test_field.cpp:52-71): max abs error 1e-4
    hg = np.array([0.532, 1.337, 1.2, 0.055], np.float32)
    fg = hg.copy()
    fg[3] = hg[3] * 2
    on_grid = lambda b: b / (128 * float(hg[3]))  # noqa: E731
    il = np.array([[0.0, 0.0], [on_grid(3), on_grid(-5)]], np.float32)
    sph = np.array([[0.0, 0.3, -0.2, 2.0, 1.36]], np.float32)
    truth_holo = O.forward_fields(sph, il, hg, 128, "born")
    truth = O.forward_fields(sph, il, fg, 64, "born")
    c = (on_grid(35), on_grid(35))
    holo = O.synthesize_holograms(truth_holo, il, hg, c)
    bg = O.synthesize_holograms(np.ones((2, 128, 128), np.complex64), il, hg, c)
    kw = dict(center=(35.0, 35.0), radius=17.0, output_size=64)
    ratio = qh.field_ratio(qh.extract_fields(holo, **kw), qh.extract_fields(bg, **kw))
    assert np.max(np.abs(ratio - truth)) < 1e-4


def test_noisy_hologram_stays_close(qh):
    # Field.NoisyHologramStaysClose (tests/test_field.cpp:88-106): noise of 2 % of the mean intensity,
    # interior rms (8-pixel margin) below 0.02.
    hg = np.array([0.532, 1.337, 1.2, 0.055], np.float32)
    fg = hg.copy()
    fg[3] = hg[3] * 2
    il = np.array([[0.0, 0.0], [0.4, -0.7]], np.float32)
    sph = np.array([[0.0, 0.3, -0.2, 2.0, 1.36]], np.float32)
    truth_holo = O.forward_fields(sph, il, hg, 128, "born")
    truth = O.forward_fields(sph, il, fg, 64, "born")
    holo = qh.synthesize_holograms(truth_holo, il, geom(qh, hg), carrier=(5.0, 5.0), noise=0.04, seed=3)
    bg = qh.synthesize_holograms(np.ones((2, 128, 128), np.complex64), il, geom(qh, hg), carrier=(5.0, 5.0),
                                 noise=0.04, seed=4)
    kw = dict(center=(35.2, 35.2), radius=17.0, output_size=64)
    ratio = qh.field_ratio(qh.extract_fields(holo, **kw), qh.extract_fields(bg, **kw))
    d = (ratio - truth)[:, 8:-8, 8:-8]
    assert float(np.sqrt(np.mean(np.abs(d) ** 2))) < 0.02


def test_auto_detection_matches_explicit_centre(qh):
    # Field.AutoDetectionMatchesExplicitCentre (tests/test_field.cpp:108-119)
    hg = np.array([0.532, 1.337, 1.2, 0.055], np.float32)
    sph = np.array([[0.0, 0.3, -0.2, 2.0, 1.36]], np.float32)
    truth = O.forward_fields(sph, np.zeros((1, 2), np.float32), hg, 128, "born")
    holo = O.synthesize_holograms(truth, np.zeros((1, 2), np.float32), hg)
    a = qh.extract_fields(holo, radius=17.0)
    b = qh.extract_fields(holo, center=(35.0, 35.0), radius=17.0)
    assert np.max(np.abs(a - b)) < 1e-6


def test_field_ratio_matches_oracle(qh):
    rng = np.random.default_rng(4)
    s = (rng.standard_normal((3, 16, 16)) + 1j * rng.standard_normal((3, 16, 16))).astype(np.complex64)
    b = (rng.standard_normal((1, 16, 16)) + 1j * rng.standard_normal((1, 16, 16)) + 3).astype(np.complex64)
    assert rel_err(qh.field_ratio(s, b), O.field_ratio(s, b)) < 1e-6
    b3 = np.concatenate([b, b * 2, b * 3])
    assert rel_err(qh.field_ratio(s, b3), O.field_ratio(s, b3)) < 1e-6
    with pytest.raises(ValueError):
        qh.field_ratio(s, b3[:2])


# ---- unwrap / Rytov ----------------------------------------------------------------------------


def test_rytov_and_unwrap_match_reference(qh):
    # Cuda.UnwrapAndRytovMatchCpu (tests/test_cuda.cpp:68-72): 1e-4 relative
    g = golden("rytov")
    assert rel_err(qh.rytov(g["ratio"]), g["rytov"]) < 1e-4
    assert rel_err(qh.unwrap(g["wrapped"]), g["unwrapped"]) < 1e-4


def _smooth_phase(nz, ny, nx):
    z, y, x = np.indices((nz, ny, nx)).astype(np.float32)
    u = (x - nx * 0.4) / (nx * 0.15)
    v = (y - ny * 0.5) / (ny * 0.2)
    w = (x - nx * 0.7) / (nx * 0.1)
    s = (y - ny * 0.3) / (ny * 0.1)
    return (30.0 * np.exp(-(u * u + v * v)) - (12.0 + z) * np.exp(-(w * w + s * s)) + 0.05 * x).astype(np.float32)


def test_unwrap_recovers_smooth_phase_up_to_constant(qh):
    # Unwrap.RecoversSmoothPhaseUpToConstant (tests/test_unwrap.cpp:34-52)
    truth = _smooth_phase(2, 96, 128)
    got = qh.unwrap(O.wrap_phase(truth))
    for z in range(2):
        offset = got[z, 0, 0] - truth[z, 0, 0]
        assert abs(math.remainder(float(offset), 2 * math.pi)) < 1e-3
        assert np.max(np.abs(got[z] - truth[z] - offset)) < 2e-3


def test_rytov_puts_border_near_zero(qh):
    # Unwrap.RytovPutsBorderNearZero (tests/test_unwrap.cpp:54-65)
    phase = _smooth_phase(1, 64, 64) + np.float32(4 * math.pi)
    ratio = (0.8 * np.exp(1j * phase.astype(np.float64))).astype(np.complex64)
    r = qh.rytov(ratio)
    assert np.max(np.abs(r.real - np.log(np.float32(0.8)))) < 1e-5
    assert np.max(np.abs(r.imag - (phase - np.float32(4 * math.pi)))) < 2e-3


@pytest.mark.parametrize("shape", [(7, 128, 128), (3, 192, 192), (2, 96, 64), (1, 384, 384), (1, 512, 512)])
def test_unwrap_sizes_match_oracle(qh, shape):
    rng = np.random.default_rng(shape[1])
    truth = _smooth_phase(*shape) + rng.normal(0, 0.1, shape).astype(np.float32)
    w = O.wrap_phase(truth)
    assert rel_err(qh.unwrap(w), O.unwrap(w)) < 1e-4


def test_unwrap_rejects_odd_sizes(qh):
    with pytest.raises(ValueError):
        qh.unwrap(np.zeros((5, 6), np.float32))


# ---- reconstruction ----------------------------------------------------------------------------


@pytest.mark.parametrize("case,kw", [("plain", {}), ("gp_r2c", dict(iterations=5)),
                                     ("gp_c2c", dict(iterations=5, gp_transform="c2c")),
                                     ("tv", dict(iterations=5, solver="tv")),
                                     ("tv_nz34", dict(iterations=3, solver="tv", nz=34))])
def test_reconstruct_api_matches_reference(qh, case, kw):
    g = golden("reconstruct")
    ri, filled = qh.reconstruct(g["fields"], g["illum"], geom(qh, g["geom"]), return_filled=True, **kw)
    assert contrast_err(ri, g[case], float(g["geom"][1])) < 1e-4
    assert filled == float(g[case + "_filled"])


def test_recovers_sphere_index_and_gp_helps(qh):
    # Odt.RecoversSphereIndexAndGpHelps (tests/test_odt.cpp:45-62), on the device.
    sph = np.array([[0.0, 0.0, 0.0, 3.0, 1.36]], np.float32)
    il = O.circular_scan(49, 0.9, G)
    fields = qh.rytov(O.forward_fields(sph, il, G, 64, "rytov"))
    truth = O.render_phantom(sph, G, 64, 64)
    plain = qh.reconstruct(fields, il, geom(qh, G))
    gp = qh.reconstruct(fields, il, geom(qh, G), iterations=20)
    tv = qh.reconstruct(fields, il, geom(qh, G), iterations=20, solver="tv")
    z, y, x = np.indices(truth.shape) - 32
    inner = (z * z + y * y + x * x) * 0.04 < 0.36 * 9.0
    rmse = lambda v: float(np.sqrt(np.mean((v.astype(np.float64) - truth) ** 2)))  # noqa: E731
    assert abs(plain[inner].mean() - 1.36) < 4e-3 and abs(gp[inner].mean() - 1.36) < 4e-3
    assert rmse(gp) < 0.7 * rmse(plain)
    # Odt.TvReducesErrorAgainstGp (tests/test_odt.cpp:88-101)
    assert abs(tv[inner].mean() - 1.36) < 4e-3 and rmse(tv) < rmse(gp)


def test_real_gp_matches_complex_gp(qh):
    # Odt.RealGpMatchesComplexGp (tests/test_odt.cpp:66-86): R2C and C2C GP iterates agree (1e-4,
    # measured 5e-6 by the reference) and fill exactly the same k-space voxels.
    sph = np.array([[0.0, 0.0, 0.0, 3.0, 1.36]], np.float32)
    il = O.circular_scan(49, 0.9, G)
    fields = qh.rytov(O.forward_fields(sph, il, G, 64, "rytov"))
    a, fa = qh.reconstruct(fields, il, geom(qh, G), iterations=10, return_filled=True)
    b, fb = qh.reconstruct(fields, il, geom(qh, G), iterations=10, gp_transform="c2c", return_filled=True)
    assert contrast_err(a, b, float(G[1])) < 1e-4
    assert fa == fb


def test_reconstruct_rejects_bad_arguments(qh):
    f = np.zeros((3, 8, 8), np.complex64)
    with pytest.raises(ValueError):
        qh.reconstruct(f, np.zeros((2, 2), np.float32), geom(qh, G))
    with pytest.raises(ValueError):
        qh.reconstruct(f, np.zeros((3, 2), np.float32), geom(qh, G), nz=7)
    with pytest.raises(ValueError):
        qh.reconstruct(f, np.full((3, 2), 10.0, np.float32), geom(qh, G))
    with pytest.raises(RuntimeError):
        qh.reconstruct(f, np.zeros((3, 2), np.float32), geom(qh, G), backend="cpu")


# ---- pipeline ----------------------------------------------------------------------------------


def test_pipeline_matches_reference_and_reuses_state(qh):
    # Pipeline.CudaMatchesCpuAndReusesPlans (tests/test_pipeline.cpp:80-97)
    g = golden("pipeline")
    for chunks in (1, 4):
        p = qh.Pipeline(5, 64, tuple(g["center"]), g["illum"], geom(qh, g["geom"]), radius=float(g["radius"]),
                        output_size=int(g["out"]), iterations=5, upload_chunks=chunks)
        p.set_background(g["bg"])
        first = p.run(g["holo"])
        assert contrast_err(first, g["ri"], float(g["geom"][1])) < 1e-4
        assert p.filled == float(g["filled"])
        second = p.run(g["holo"])
        assert np.array_equal(first, second)
        assert p.device_bytes > 0 and p.timings["total"] > 0 and p.setup_ms > 0


def test_pipeline_needs_background_and_carrier(qh):
    # Pipeline.NeedsBackgroundAndCarrier (tests/test_pipeline.cpp:72-78)
    il = O.circular_scan(3, 0.9, G)
    p = qh.Pipeline(3, 32, (8, 8), il, geom(qh, G), output_size=16)
    with pytest.raises(RuntimeError):
        p.run(np.zeros((3, 32, 32), np.float32))
    with pytest.raises(ValueError):
        qh.Pipeline(3, 32, (8, 8), il, geom(qh, G), output_size=16, upload_chunks=4)


def test_pipeline_tv_matches_per_call_chain(qh):
    # python/tests/test_qoraholo.py:235-257, with the FISTA-TV solver.
    hg = np.array([0.532, 1.337, 1.2, 0.1], np.float32)
    il = O.circular_scan(9, 0.9, G)
    sph = np.array([[0.0, 0.0, 0.0, 3.0, 1.36]], np.float32)
    ratio = O.forward_fields(sph, il, hg, 128)
    c = 36 / (128 * 0.1)
    holo = O.synthesize_holograms(ratio, il, hg, carrier=(c, c))
    bg = O.synthesize_holograms(np.ones_like(ratio), il, hg, carrier=(c, c))
    crop = dict(center=(36, 36), radius=30, output_size=64)
    fields = qh.field_ratio(qh.extract_fields(holo, **crop), qh.extract_fields(bg, **crop))
    ref = qh.reconstruct(qh.rytov(fields), il, geom(qh, G), iterations=3, solver="tv")
    p = qh.Pipeline(9, 128, illuminations=il, geometry=geom(qh, G), iterations=3, solver="tv", **crop)
    p.set_background(bg)
    ri = p.run(holo)
    assert contrast_err(ri, ref, 1.337) < 1e-4
    cref = O.reconstruct(O.rytov(O.field_ratio(O.extract_fields(holo, **crop), O.extract_fields(bg, **crop))), il, G,
                         iterations=3, solver="tv")[0]
    assert contrast_err(ri, cref, 1.337) < 1e-4


# ---- BPM ---------------------------------------------------------------------------------------


def test_bpm_forward_matches_reference(qh):
    g = golden("bpm")
    assert rel_err(qh.bpm_forward(g["ri"], g["illum"], geom(qh, G)) - 1, g["forward"] - 1) < 1e-4


def test_bpm_vjp_matches_reference(cuda):
    from qoraholo_b200 import capi

    g = golden("bpm")
    xc = (g["ri"] - G[1]).astype(np.float32)
    assert rel_err(capi.bpm_vjp(xc, g["residual"], g["illum"], G), g["vjp"]) < 1e-4


@pytest.mark.parametrize("batch", [0, 2])
def test_bpm_reconstruct_matches_reference(qh, batch):
    # Cuda.BpmReconstructionMatchesCpu (tests/test_cuda.cpp:163-182): 1e-3
    g = golden("bpm")
    init = np.full((16, 24, 24), G[1], np.float32)
    ri, loss = qh.bpm_reconstruct(g["forward"], g["illum"], geom(qh, G), init, iterations=3, batch=batch,
                                  tv_weight=1e-2, return_loss=True)
    assert contrast_err(ri, g[f"rec_batch{batch}"], G[1]) < 1e-3
    np.testing.assert_allclose(loss[-1], g[f"loss_batch{batch}"][-1], rtol=1e-3)


def test_bpm_matches_oracle_larger(qh):
    # Cuda.BpmMatchesCpu (tests/test_cuda.cpp:140-146) at 32 x 48^2, 7 angles.
    il = O.circular_scan(7, 0.9, G)
    ri = O.render_phantom(CELL, G, 32, 48)
    assert rel_err(qh.bpm_forward(ri, il, geom(qh, G)) - 1, O.bpm_forward(ri, il, G) - 1) < 1e-4


def test_bpm_inverts_exact_bead(qh):
    # python/tests/test_qoraholo.py:106-115
    bead = np.array([[0.0, 0.0, 0.0, 3.0, 1.40]], np.float32)
    il = O.circular_scan(25, 0.9, G)
    data = O.forward_fields(bead, il, G, 64, "exact")
    initial = qh.reconstruct(qh.rytov(data), il, geom(qh, G), iterations=10)
    ri, loss = qh.bpm_reconstruct(data, il, geom(qh, G), initial, iterations=10, return_loss=True)
    assert ri.shape == (64, 64, 64) and loss.shape == (10,) and loss[-1] < loss[0]
    truth = O.render_phantom(bead, G, 64, 64)
    assert np.sqrt(np.mean((ri - truth) ** 2)) < np.sqrt(np.mean((initial - truth) ** 2))


# ---- fixture generators ------------------------------------------------------------------------


def test_phantom_generators_match_reference(qh):
    g = golden("phantom")
    gg = geom(qh, G)
    assert rel_err(qh.forward_fields(spheres(qh, CELL), g["illum"], gg, 32, "born") - 1, g["born"] - 1) < 1e-5
    assert rel_err(qh.forward_fields(spheres(qh, CELL), g["illum"], gg, 32) - 1, g["rytov"] - 1) < 1e-5
    assert rel_err(qh.forward_fields(spheres(qh, CELL[:1]), g["illum"], gg, 32, "exact") - 1, g["exact"] - 1) < 1e-5
    np.testing.assert_array_equal(qh.render_phantom(spheres(qh, CELL), gg, 12, 32), g["render"])
    np.testing.assert_allclose(qh.synthesize_holograms(g["rytov"], g["illum"], gg, (1.0, 1.5)), g["holo"], rtol=1e-6)
    np.testing.assert_array_equal(qh.circular_scan(49, 0.9, gg), g["scan49"])


# ---- hologram synthesis on the device ---------------------------------------------------------


def test_device_holograms_match_host_synthesis(qh):
    """synthesize_holograms on the device (src/phantom.cpp:193-221): noise-free intensities equal the
    host's to float rounding; the noise has the requested mean and spread, is reproducible for a seed
    and changes with it."""
    import torch

    from qoraholo_b200 import capi

    hg = np.array([0.532, 1.337, 1.2, 0.1], np.float32)
    il = O.circular_scan(5, 0.9, G)
    ratio = O.forward_fields(np.array([[0.0, 0.3, -0.2, 2.0, 1.36]], np.float32), il, hg, 96)
    c = (30 / (96 * 0.1), 28 / (96 * 0.1))
    host = qh.synthesize_holograms(ratio, il, geom(qh, hg), carrier=c)
    d_ratio = torch.from_numpy(np.ascontiguousarray(ratio, np.complex64)).cuda()
    out = torch.empty((5, 96, 96), dtype=torch.float32, device="cuda")

    def run(noise, seed):
        capi.synthesize_holograms_device(d_ratio.data_ptr(), 5, 96, il, float(hg[3]), carrier=c, noise=noise,
                                         seed=seed, d_out=out.data_ptr())
        return out.cpu().numpy()

    clean = run(0.0, 1)
    assert rel_err(clean, host) < 1e-6
    noisy = run(0.02, 7)
    d = (noisy - clean).astype(np.float64)
    assert abs(d.mean()) < 3 * 0.02 / np.sqrt(d.size) + 1e-6
    assert abs(d.std() - 0.02) < 0.02 * 0.02
    assert np.array_equal(noisy, run(0.02, 7))
    assert not np.array_equal(noisy, run(0.02, 8))
