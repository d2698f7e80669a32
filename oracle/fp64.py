"""FP64 restatement of the reference's hologram -> refractive-index path (field extraction, ratio,
least-squares unwrap and Rytov, Ewald mapping, Gerchberg-Papoulis or FISTA-TV, index), every
operation in double precision, and the analytic phantom the reconstructions are scored against.

TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / parity leg
may import this module. It is the yardstick for "error against an FP64 run": the reference computes
in float32 (cfloat = std::complex<float>, include/qoraholo/array.hpp:10), and so does the CUDA path;
both are compared with this run of the same algorithm in exact-as-possible arithmetic.

The algorithm follows the float32 oracle (oracle/qh_oracle.py) and the reference functions it cites:
src/cpu/field.cpp:78-121 (fields), src/cpu/field.cpp:62-74 (ratio), src/cpu/unwrap.cpp:11-82 with the
DCT of src/cpu/fft.cpp:101-133 (unwrap, Rytov), src/common.hpp:56-87 and src/cpu/odt.cpp:124-242
(mapping, Hermitian half data, GP and FISTA-TV loops), src/cpu/tv.cpp:7-44 (FGP, in oracle/fp64_tv.c)
and src/common.hpp:179-183 (index). The Ewald bins are chosen in double too, so a bin whose float32
index rounds the other way counts as part of the float32 error. The DCT pair is scipy's (an exact
inverse pair), which solves the same Neumann least-squares problem as the reference's Makhoul DCT.
"""

from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import scipy.fft as sfft

HERE = Path(__file__).resolve().parent
LIB = HERE / "_fp64" / "libqhfp64.so"
SRC = HERE / "fp64_tv.c"
WORKERS = -1
_lib = None


def build(force: bool = False) -> Path | None:
    """Compiles oracle/fp64_tv.c into oracle/_fp64/libqhfp64.so (gcc, OpenMP) when it is stale."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    try:
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", str(LIB), str(SRC), "-lm"])
    except (OSError, subprocess.CalledProcessError):
        return LIB if LIB.exists() else None
    return LIB


def lib():
    global _lib
    if _lib is None:
        if build() is None:
            raise FileNotFoundError(f"{LIB} is not built and gcc is not available")
        _lib = C.CDLL(str(LIB))
        _lib.fp64_tv_prox.restype = C.c_int
        _lib.fp64_tv_prox.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                      C.c_void_p]
        _lib.fp64_threads.restype = C.c_int
    return _lib


def threads() -> int:
    return int(lib().fp64_threads())


def _parity(i):
    return np.where(np.asarray(i) & 1, -1.0, 1.0)


def _signed_bin(k, n):
    k = np.asarray(k)
    return np.where(k < n // 2, k, k - n)


# ---------------------------------------------------------------------------------------------
# fields, ratio, unwrap, Rytov


def extract_fields(holograms, center, radius, output_size):
    """Sideband crop in centre-origin bookkeeping, in double (src/cpu/field.cpp:78-121)."""
    h = np.asarray(holograms, np.float64)
    if h.ndim == 2:
        h = h[None]
    n = h.shape[-1]
    cy, cx = (int(math.floor(abs(float(c)) + 0.5)) * (1 if float(c) >= 0 else -1) for c in center)
    m = int(output_size)
    yy, xx = np.indices((n, n))
    spec = sfft.fft2(h * _parity(yy + xx), workers=WORKERS)
    dy = (np.arange(m) - m // 2)[:, None]
    dx = (np.arange(m) - m // 2)[None, :]
    sy, sx = n // 2 + cy + dy, n // 2 + cx + dx
    inside = ((dy * dy + dx * dx) <= float(radius) ** 2) & (sy >= 0) & (sy < n) & (sx >= 0) & (sx < n)
    out = np.zeros((h.shape[0], m, m), np.complex128)
    iy, ix = np.nonzero(inside)
    out[:, iy, ix] = spec[:, sy[iy, 0], sx[0, ix]] * _parity(cy + cx)
    out = sfft.ifft2(out, workers=WORKERS) * (float(m * m) / float(n * n))
    y, x = np.indices((m, m))
    return out * _parity(x + y)


def field_ratio(sample, background):
    return np.asarray(sample, np.complex128) / np.asarray(background, np.complex128)


def _wrap(p):
    return p - 2.0 * math.pi * np.floor((p + math.pi) / (2.0 * math.pi))


def unwrap(psi):
    """Least-squares unwrap (Neumann Poisson by DCT) plus the congruence constant
    (src/cpu/unwrap.cpp:11-59), in double."""
    psi = np.asarray(psi, np.float64)
    if psi.ndim == 2:
        psi = psi[None]
    _, ny, nx = psi.shape
    dxp = _wrap(psi[:, :, 1:] - psi[:, :, :-1])
    dyp = _wrap(psi[:, 1:, :] - psi[:, :-1, :])
    rho = np.zeros_like(psi)
    rho[:, :, :-1] += dxp
    rho[:, :, 1:] -= dxp
    rho[:, :-1, :] += dyp
    rho[:, 1:, :] -= dyp
    d = sfft.dctn(rho, type=2, axes=(1, 2), workers=WORKERS)
    ky = np.arange(ny)[:, None]
    kx = np.arange(nx)[None, :]
    ev = 2.0 * np.cos(math.pi * ky / ny) + 2.0 * np.cos(math.pi * kx / nx) - 4.0
    ev[0, 0] = 1.0
    d = d / ev
    d[:, 0, 0] = 0.0
    phi = sfft.idctn(d, type=2, axes=(1, 2), workers=WORKERS)
    acc = np.exp(1j * (psi - phi)).reshape(psi.shape[0], -1).sum(axis=1)
    return phi + np.angle(acc)[:, None, None]


def rytov(ratio):
    """log|r| + i (unwrap(arg r) - 2 pi m), m from the border mean (src/cpu/unwrap.cpp:61-82)."""
    r = np.asarray(ratio, np.complex128)
    if r.ndim == 2:
        r = r[None]
    _, ny, nx = r.shape
    phase = unwrap(np.angle(r))
    border = (phase[:, 0, :].sum(1) + phase[:, ny - 1, :].sum(1) + phase[:, 1:ny - 1, 0].sum(1)
              + phase[:, 1:ny - 1, nx - 1].sum(1))
    mean = border / (2.0 * nx + 2.0 * (ny - 2))
    shift = 2.0 * math.pi * np.round(mean / (2.0 * math.pi))
    return np.log(np.abs(r)) + 1j * (phase - shift[:, None, None])


# ---------------------------------------------------------------------------------------------
# ODT


def _grid(n, nz, geom):
    wavelength, n_medium, na, pixel = (float(v) for v in geom)
    fm, fna = n_medium / wavelength, na / wavelength
    return dict(n=n, nz=nz, df=1.0 / (n * pixel), dfz=1.0 / (nz * pixel), fm2=fm * fm, fna2=fna * fna,
                gain=4.0 * math.pi / pixel)


def ewald_map(spectra, illuminations, g):
    """Column-owner mapping in illumination order (src/cpu/odt.cpp:137-171), bins chosen in double.
    Returns the normalised potential (nz, n, n) and the hit weights."""
    n, nz = g["n"], g["nz"]
    il = np.asarray(illuminations, np.float64).reshape(-1, 2)
    pot = np.zeros((nz, n, n), np.complex128)
    weight = np.zeros((nz, n, n), np.float64)
    sb = _signed_bin(np.arange(n), n) * g["df"]
    yy, xx = np.indices((n, n))
    for a in range(il.shape[0]):
        fiy, fix = il[a]
        fiz = math.sqrt(g["fm2"] - fiy * fiy - fix * fix)
        fy, fx = (sb + fiy)[:, None], (sb + fix)[None, :]
        rho2 = fy * fy + fx * fx
        ok = ~((rho2 > g["fna2"]) | (rho2 >= g["fm2"]))
        nuz = np.sqrt(np.where(ok, g["fm2"] - rho2, 0.0))
        k = np.floor((nuz - fiz) / g["dfz"] + 0.5).astype(np.int64)
        ok &= (k >= -(nz // 2)) & (k < nz // 2)
        kz = np.where(k < 0, k + nz, k)
        v = (-1j * g["gain"] * nuz) * spectra[a] * _parity(kz)
        sel = np.nonzero(ok)
        np.add.at(pot, (kz[sel], yy[sel], xx[sel]), v[sel])
        np.add.at(weight, (kz[sel], yy[sel], xx[sel]), 1.0)
    filled = weight > 0
    pot[filled] /= weight[filled]
    return pot, weight


def _half(pot, weight):
    """Hermitian half data and hit counts (src/common.hpp:70-87, src/cpu/odt.cpp:37-62)."""
    nz, n, _ = pot.shape
    h = n // 2 + 1
    mz, my, mx = (-np.arange(nz)) % nz, (-np.arange(n)) % n, (-np.arange(h)) % n
    neg = pot[mz][:, my][:, :, mx]
    a = 0.5 * (pot[:, :, :h].real + neg.real) + 0.5j * (pot[:, :, :h].imag - neg.imag)
    hits = (weight[:, :, :h] > 0).astype(np.int64) + (weight[mz][:, my][:, :, mx] > 0).astype(np.int64)
    return a, hits


def _restore(e, a, hits):
    return a + (1.0 - 0.5 * hits) * e


def _irfft3(e, shape):
    return sfft.irfftn(e, s=shape, axes=(0, 1, 2), workers=WORKERS)


def _rfft3(x):
    return sfft.rfftn(x, axes=(0, 1, 2), workers=WORKERS)


def tv_prox(b, p, lam, inner):
    """FGP (oracle/fp64_tv.c); p (3, nz, ny, nx) float64, updated in place."""
    b = np.ascontiguousarray(b, np.float64)
    assert p.dtype == np.float64 and p.flags.c_contiguous and p.shape == (3,) + b.shape
    x = np.empty_like(b)
    nz, ny, nx = b.shape
    code = lib().fp64_tv_prox(b.ctypes.data, p.ctypes.data, nz, ny, nx, float(lam), int(inner), x.ctypes.data)
    if code:
        raise RuntimeError(f"fp64_tv_prox failed ({code})")
    return x


def reconstruct(fields, illuminations, geom, nz=0, iterations=0, solver="gp", tv_weight=1e-2, tv_inner=10):
    """Rytov ODT with the R2C Gerchberg-Papoulis or FISTA-TV solver (src/cpu/odt.cpp:124-206) in
    double. Returns (index volume float64, filled fraction)."""
    f = np.asarray(fields, np.complex128)
    if f.ndim == 2:
        f = f[None]
    count, _, n = f.shape
    nz = nz or n
    g = _grid(n, nz, geom)
    spectra = sfft.fft2(f, workers=WORKERS)
    pot, weight = ewald_map(spectra, illuminations, g)
    filled = float(np.count_nonzero(weight)) / weight.size
    k0 = 2.0 * math.pi / float(geom[0])
    nm2 = float(geom[1]) ** 2
    shape = (nz, n, n)
    if iterations > 0:
        a, hits = _half(pot, weight)
        del pot, weight
        y = _irfft3(a, shape)
        if solver == "tv":
            lam = float(tv_weight) * k0 * k0
            x_prev = y.copy()
            p = np.zeros((3,) + shape, np.float64)
            t = 1.0
            for _ in range(iterations):
                y = _irfft3(_restore(_rfft3(y), a, hits), shape)
                x = tv_prox(y, p, lam, tv_inner)
                t_next = 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t))
                y = x + (t - 1.0) / t_next * (x - x_prev)
                x_prev, t = x, t_next
            x = x_prev
        else:
            x = y
            for _ in range(iterations):
                x = _irfft3(_restore(_rfft3(np.maximum(x, 0.0)), a, hits), shape)
        re, im = x, 0.0
    else:
        v = sfft.ifftn(pot, axes=(0, 1, 2), workers=WORKERS)
        re, im = v.real, v.imag
    aa = nm2 + re / (k0 * k0)
    bb = im / (k0 * k0)
    return np.sqrt(0.5 * (np.hypot(aa, bb) + aa)), filled


def pipeline(holograms, backgrounds, center, radius, output_size, illuminations, geom, **solver):
    """Pipeline::process (src/pipeline.cpp:116-129) in double: fields of holograms and backgrounds,
    their ratio, Rytov, reconstruct. Returns (index volume, filled)."""
    u = extract_fields(holograms, center, radius, output_size)
    ub = extract_fields(backgrounds, center, radius, output_size)
    return reconstruct(rytov(field_ratio(u, ub)), illuminations, geom, **solver)


# ---------------------------------------------------------------------------------------------
# analytic phantom


def render_ellipsoids(shapes, n_medium, pixel, nz, n):
    """Index volume of nested ellipsoids in painter's order on the reconstruction grid: voxel
    (k, j, i) sits at ((k - nz/2), (j - n/2), (i - n/2)) * pixel (src/phantom.cpp:84-100 for
    spheres). shapes: (centre (z, y, x), semi-axes (z, y, x), index) triples."""
    k, j, i = np.indices((nz, n, n), dtype=np.float64)
    z, y, x = (k - nz // 2) * pixel, (j - n // 2) * pixel, (i - n // 2) * pixel
    out = np.full((nz, n, n), float(n_medium))
    for c, a, idx in shapes:
        inside = ((z - c[0]) / a[0]) ** 2 + ((y - c[1]) / a[1]) ** 2 + ((x - c[2]) / a[2]) ** 2 <= 1.0
        out[inside] = float(idx)
    return out


def rmse(a, b):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    return float(np.sqrt(np.mean(d * d)))


def rel_contrast_err(a, ref, n_medium):
    """|a - ref| / |ref - n_medium|, the index-contrast error of the reference's tests
    (tests/test_cuda.cpp:92-97)."""
    a = np.asarray(a, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.linalg.norm(a - ref) / np.linalg.norm(ref - float(n_medium)))
