"""Writes the golden fixtures in this folder: inputs and outputs of the reference's own CPU
implementation (oracle/_ref/libqhref.so, built from the reference sources by
oracle/build_ref.py), on small versions of the cases its test suite checks (tests/test_dct.cpp,
test_field.cpp, test_unwrap.cpp, test_odt.cpp, test_cuda.cpp, test_bpm.cpp, test_pipeline.cpp).

Run in a container that has the reference sources:  python tests/golden/make_golden.py
The fixtures are committed; the tests only read them.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import build_ref, refimpl as R  # noqa: E402

GEOM = np.array([0.532, 1.337, 1.2, 0.2], np.float32)
CELL = np.array([[0.0, 0.4, -0.3, 2.5, 1.36], [0.0, 0.4, -0.3, 1.0, 1.38]], np.float32)


def save(name, **arrays):
    np.savez_compressed(HERE / f"{name}.npz", **arrays)


def main():
    build_ref.build()
    # Dct.MatchesPocketfftTypeTwo / InverseRoundTrips (tests/test_dct.cpp:22-47)
    rng = np.random.default_rng(7)
    a = rng.uniform(-1, 1, (3, 12, 10)).astype(np.float32)
    save("dct", a=a, dct_y=R.dct2(a, 1), dct_x=R.dct2(a, 2), idct_y=R.dct2(a, 1, True),
         idct_x=R.dct2(a, 2, True), pocket_y=R.pocketfft_dct2(a, 1, 0.5), pocket_x=R.pocketfft_dct2(a, 2, 0.5))

    # Cuda.FieldExtractionMatchesCpu / AcrossZeroKx (tests/test_cuda.cpp:37-66)
    hg = GEOM.copy()
    hg[3] = 0.05
    il = R.circular_scan(3, 0.8, GEOM)
    holo = R.synthesize_holograms(R.forward_fields(CELL, il, hg, 128, "rytov"), il, hg, (5.0, 5.0), 1.0, 0.02, 1)
    save("field", holo=holo, center=np.array([32.0, 32.0], np.float32), radius=np.float32(16.0), out=np.int32(64),
         fields=R.extract_fields(holo, (32.0, 32.0), 16.0, 0.0, 64))
    df = np.float32(1.0) / (np.float32(128) * hg[3])
    il3 = R.circular_scan(3, 0.5, GEOM)
    holo = R.synthesize_holograms(R.forward_fields(CELL, il3, hg, 128, "rytov"), il3, hg,
                                  (-30.0 * df, 4.0 * df), 1.0, 0.02, 1)
    save("field_negkx", holo=holo, center=np.array([-30.0, 4.0], np.float32), radius=np.float32(12.0),
         out=np.int32(32), fields=R.extract_fields(holo, (-30.0, 4.0), 12.0, 0.0, 32))

    # Field.FindsCarrierSideband (tests/test_field.cpp:39-50)
    g55 = np.array([0.532, 1.337, 1.2, 0.055], np.float32)
    bg = R.synthesize_holograms(np.ones((1, 128, 128), np.complex64), np.zeros((1, 2), np.float32), g55,
                                (5.0, 5.0), 1.0, 0.0, 1)
    iy, ix, y, x, mag = R.find_sideband(bg)
    save("sideband", holo=bg, iy=np.int32(iy), ix=np.int32(ix), y=np.float32(y), x=np.float32(x),
         magnitude=np.float32(mag))

    # Cuda.UnwrapAndRytovMatchCpu (tests/test_cuda.cpp:68-72); Unwrap.* (tests/test_unwrap.cpp)
    il5 = R.circular_scan(5, 0.8, GEOM)
    ratio = R.forward_fields(CELL, il5, GEOM, 48, "rytov")
    z, y, x = np.indices((2, 32, 48)).astype(np.float32)
    u = (x - 48 * 0.4) / (48 * 0.15)
    v = (y - 32 * 0.5) / (32 * 0.2)
    w = (x - 48 * 0.7) / (48 * 0.1)
    s = (y - 32 * 0.3) / (32 * 0.1)
    truth = (30.0 * np.exp(-(u * u + v * v)) - (12.0 + z) * np.exp(-(w * w + s * s)) + 0.05 * x).astype(np.float32)
    wrapped = np.angle(np.exp(1j * truth.astype(np.float64))).astype(np.float32)
    save("rytov", ratio=ratio, rytov=R.rytov(ratio), wrapped=wrapped, unwrapped=R.unwrap(wrapped))

    # Cuda.ReconstructionMatchesCpu / TvMatchesCpu (tests/test_cuda.cpp:74-115), at 32^3
    g3 = GEOM.copy()
    g3[3] = 0.3
    il13 = R.circular_scan(13, 0.9, g3)
    fields = R.rytov(R.forward_fields(CELL, il13, g3, 32, "rytov"))
    cases = {}
    for name, kw in [("plain", {}), ("gp_r2c", dict(iterations=5)), ("gp_c2c", dict(iterations=5, gp_transform="c2c")),
                     ("tv", dict(iterations=5, solver="tv")), ("tv_nz34", dict(iterations=3, solver="tv", nz=34))]:
        ri, filled = R.reconstruct(fields, il13, g3, **kw)
        cases[name] = ri
        cases[name + "_filled"] = np.float64(filled)
    save("reconstruct", fields=fields, illum=il13, geom=g3, **cases)

    # cpu::tv_prox (src/cpu/tv.cpp:7-44), warm-started dual
    rng = np.random.default_rng(3)
    b = rng.uniform(-0.2, 1.0, (10, 12, 20)).astype(np.float32)
    p0 = (rng.uniform(-0.5, 0.5, (3, 10, 12, 20)) * (rng.uniform(size=(3, 10, 12, 20)) > 0.5)).astype(np.float32)
    x, p = R.tv_prox(b, p0, 0.05, 7)
    save("tv_prox", b=b, p0=p0, lam=np.float32(0.05), inner=np.int32(7), x=x, p=p)

    # Cuda.Bpm* (tests/test_cuda.cpp:140-196), at 16 x 24 x 24
    il7 = R.circular_scan(5, 0.9, GEOM)
    ri = R.render_phantom(CELL, GEOM, 16, 24)
    fwd = R.bpm_forward(ri, il7, GEOM)
    xc = (ri - np.float32(GEOM[1])).astype(np.float32)
    idx = np.arange(5 * 24 * 24)
    r = (np.sin(0.7 * idx) + 1j * np.cos(1.3 * idx)).astype(np.complex64).reshape(5, 24, 24)
    vjp = R.bpm_vjp(xc, r, il7, GEOM)
    init = np.full((16, 24, 24), GEOM[1], np.float32)
    rec0, loss0 = R.bpm_reconstruct(fwd, il7, GEOM, init, iterations=3, batch=0, tv_weight=1e-2)
    rec2, loss2 = R.bpm_reconstruct(fwd, il7, GEOM, init, iterations=3, batch=2, tv_weight=1e-2)
    save("bpm", ri=ri, illum=il7, forward=fwd, residual=r, vjp=vjp, rec_batch0=rec0, loss_batch0=loss0,
         rec_batch2=rec2, loss_batch2=loss2)

    # Pipeline.CpuMatchesPerCallFunctions (tests/test_pipeline.cpp:62-70), at 64^2 -> 32^3
    hg2 = GEOM.copy()
    hg2[3] = 0.15
    g2 = GEOM.copy()
    g2[3] = 0.3
    il9 = R.circular_scan(5, 0.9, g2)
    dfp = np.float32(1.0) / (np.float32(64) * hg2[3])
    ratio = R.forward_fields(CELL, il9, hg2, 64, "rytov")
    holo = R.synthesize_holograms(ratio, il9, hg2, (18.0 * dfp, 18.0 * dfp), 1.0, 0.01, 3)
    bgh = R.synthesize_holograms(np.ones_like(ratio), il9, hg2, (18.0 * dfp, 18.0 * dfp), 1.0, 0.01, 3)
    out, filled, _ = R.pipeline(holo, bgh, (18.0, 18.0), 14.0, 32, il9, g2, iterations=5)
    save("pipeline", holo=holo, bg=bgh, illum=il9, geom=g2, center=np.array([18.0, 18.0], np.float32),
         radius=np.float32(14.0), out=np.int32(32), ri=out, filled=np.float64(filled))

    # fixture generators (src/phantom.cpp), noise-free
    il4 = R.circular_scan(4, 0.9, GEOM)
    save("phantom", illum=il4, born=R.forward_fields(CELL, il4, GEOM, 32, "born"),
         rytov=R.forward_fields(CELL, il4, GEOM, 32, "rytov"),
         exact=R.forward_fields(CELL[:1], il4, GEOM, 32, "exact"),
         render=R.render_phantom(CELL, GEOM, 12, 32),
         holo=R.synthesize_holograms(R.forward_fields(CELL, il4, GEOM, 32, "rytov"), il4, GEOM, (1.0, 1.5), 1.0, 0.0, 1),
         scan49=R.circular_scan(49, 0.9, GEOM))


if __name__ == "__main__":
    main()
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)
