"""The FP64 restatement (oracle/fp64.py, oracle/fp64_tv.c) against the float32 oracle and the
reference's own outputs (golden fixtures made by oracle/_ref): a double-precision run of the same
algorithm must sit within float32 rounding of the reference, since it is the yardstick that every
float32 result's "error against FP64" is measured with. CPU only."""

from __future__ import annotations

import numpy as np

from conftest import golden
from oracle import fp64
from oracle import qh_oracle as O


def test_fgp_in_double_tracks_the_float32_iteration():
    z = golden("tv_prox")
    p = np.ascontiguousarray(z["p0"], np.float64)
    x = fp64.tv_prox(z["b"].astype(np.float64), p, float(z["lam"]), int(z["inner"]))
    assert np.linalg.norm(x - z["x"]) / np.linalg.norm(x) < 1e-5
    assert np.linalg.norm(p - z["p"]) / np.linalg.norm(p) < 1e-5


def test_unwrap_in_double_recovers_a_smooth_phase():
    y, x = np.indices((64, 48))
    phi = (0.002 * (x - 20) ** 2 + 0.003 * (y - 30) ** 2 + 0.05 * x)[None]
    u = fp64.unwrap(np.angle(np.exp(1j * phi)))
    d = u - phi
    assert d.max() - d.min() < 1e-9  # exact up to one constant
    assert abs(d.mean()) < 1e-9      # which the congruence step removes


def test_pipeline_in_double_matches_the_reference_within_float32_error():
    z = golden("pipeline")
    ri, filled = fp64.pipeline(z["holo"], z["bg"], tuple(z["center"]), float(z["radius"]), int(z["out"]), z["illum"],
                               z["geom"], iterations=5)
    err = fp64.rel_contrast_err(z["ri"], ri, z["geom"][1])
    assert err < 1e-4, err  # the reference's float32 result against exact arithmetic
    assert abs(filled - float(z["filled"])) < 2e-3  # bins chosen in double may differ at a few edges


def test_solvers_in_double_match_the_float32_oracle():
    z = golden("reconstruct")
    for key, kw in (("gp_r2c", dict(iterations=5, solver="gp")), ("tv", dict(iterations=3, solver="tv", tv_inner=4))):
        ri, _ = fp64.reconstruct(z["fields"], z["illum"], z["geom"], **kw)
        ref, _ = O.reconstruct(z["fields"], z["illum"], z["geom"], **kw)
        assert fp64.rel_contrast_err(ref, ri, z["geom"][1]) < 1e-4


def test_rendered_ellipsoids_follow_painters_order():
    shapes = [((0.0, 0.0, 0.0), (1.0, 1.2, 1.4), 1.36), ((0.0, 0.0, 0.0), (0.4, 0.4, 0.4), 1.38)]
    v = fp64.render_ellipsoids(shapes, 1.337, 0.1, 32, 32)
    assert v[16, 16, 16] == 1.38                  # centre: the later, inner shape
    assert v[16, 16, 16 + 10] == 1.36             # 1.0 um along x: inside the body only
    assert v[0, 0, 0] == 1.337                    # corner: medium
    assert fp64.rmse(v, v) == 0.0
