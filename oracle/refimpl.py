"""ctypes access to oracle/_ref/libqhref.so, the reference's own CPU implementation built by
oracle/build_ref.py. Test infrastructure: used by tests/ (to pin the numpy oracle and to make the
golden fixtures) and by bench.py's reference arm and CPU baseline, never by the product.

Each function takes and returns numpy arrays with the reference's Python conventions
(python/qoraholo/__init__.py): float32 images / volumes, complex64 fields, (count, 2) float32
illuminations (fy, fx), and a geometry as (wavelength, n_medium, na, pixel).
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libqhref.so"
LIB_CUDA_PATH = Path(__file__).resolve().parent / "_ref" / "libqhref_cuda.so"
_lib = None
_path = LIB_PATH

_ERRORS = {1: ValueError, 2: RuntimeError, 3: RuntimeError, 4: RuntimeError}


class ReferenceLogicError(RuntimeError):
    """std::logic_error raised by the reference (e.g. process() before set_background())."""


def available() -> bool:
    return LIB_PATH.exists()


def cuda_available() -> bool:
    """The reference built with its CUDA backend (oracle/build_ref.py build_cuda) is present."""
    return LIB_CUDA_PATH.exists()


def select(cuda: bool = False):
    """Routes every call of this module to the reference's CUDA backend (reconstruct and the Pipeline
    on the GPU, src/cuda/*) or back to its CPU backend."""
    global _lib, _path
    path = LIB_CUDA_PATH if cuda else LIB_PATH
    if path != _path:
        _lib, _path = None, path
    _check(lib().ref_use_cuda(C.c_int(1 if cuda else 0)))


def lib():
    global _lib
    if _lib is None:
        if not _path.exists():
            raise FileNotFoundError(f"{_path} is not built; run python oracle/build_ref.py")
        _lib = C.CDLL(str(_path))
        _lib.ref_last_error.restype = C.c_char_p
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(code):
    if code:
        msg = lib().ref_last_error().decode()
        if code == 3:
            raise ReferenceLogicError(msg)
        raise _ERRORS.get(code, RuntimeError)(msg)


def _geom(g):
    return np.ascontiguousarray(g, np.float32).reshape(4)


def _illum(il):
    return np.ascontiguousarray(np.reshape(il, (-1, 2)), np.float32)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _c64(a):
    return np.ascontiguousarray(a, np.complex64)


def threads() -> int:
    return int(lib().ref_threads())


def circular_scan(count, na_illumination, geom):
    out = np.zeros((count, 2), np.float32)
    _check(lib().ref_circular_scan(C.c_int(count), C.c_float(na_illumination), _p(_geom(geom)), _p(out)))
    return out


def find_sideband(holograms, dc_exclusion=0.0):
    h = _f32(holograms)
    if h.ndim == 2:
        h = h[None]
    iy, ix = C.c_int(), C.c_int()
    rest = np.zeros(3, np.float32)
    _check(lib().ref_find_sideband(_p(h), C.c_int(h.shape[0]), C.c_int(h.shape[2]), C.c_float(dc_exclusion),
                                   C.byref(iy), C.byref(ix), _p(rest)))
    return iy.value, ix.value, float(rest[0]), float(rest[1]), float(rest[2])


def extract_fields(holograms, center=None, radius=0.0, dc_exclusion=0.0, output_size=0):
    h = _f32(holograms)
    nz, n = h.shape[0], h.shape[2]
    m = output_size if output_size > 0 else n
    out = np.zeros((nz, m, m), np.complex64)
    cy, cx = center if center is not None else (0.0, 0.0)
    _check(lib().ref_extract_fields(_p(h), C.c_int(nz), C.c_int(n), C.c_int(center is not None),
                                    C.c_float(cy), C.c_float(cx), C.c_float(radius), C.c_float(dc_exclusion),
                                    C.c_int(output_size), _p(out)))
    return out


def field_ratio(sample, background):
    s, b = _c64(sample), _c64(background)
    out = np.zeros_like(s)
    _check(lib().ref_field_ratio(_p(s), *map(C.c_int, s.shape), _p(b), C.c_int(b.shape[0]), _p(out)))
    return out


def unwrap(wrapped):
    w = _f32(wrapped)
    out = np.zeros_like(w)
    _check(lib().ref_unwrap(_p(w), *map(C.c_int, w.shape), _p(out)))
    return out


def rytov(ratio):
    r = _c64(ratio)
    out = np.zeros_like(r)
    _check(lib().ref_rytov(_p(r), *map(C.c_int, r.shape), _p(out)))
    return out


def dct2(a, axis, inverse=False):
    out = _f32(a).copy()
    _check(lib().ref_dct2(_p(out), *map(C.c_int, out.shape), C.c_int(axis), C.c_int(int(inverse))))
    return out


def pocketfft_dct2(a, axis, fct=1.0):
    a = _f32(a)
    out = np.zeros_like(a)
    _check(lib().ref_pocketfft_dct2(_p(a), *map(C.c_int, a.shape), C.c_int(axis), C.c_float(fct), _p(out)))
    return out


SOLVERS = {"gp": 0, "tv": 1}
TRANSFORMS = {"r2c": 0, "c2c": 1}


def reconstruct(fields, illuminations, geom, nz=0, iterations=0, solver="gp", gp_transform="r2c",
                tv_weight=1e-2, tv_inner=10, return_stages=False):
    f = _c64(fields)
    count, n = f.shape[0], f.shape[2]
    il = _illum(illuminations)
    nzz = nz if nz > 0 else n
    out = np.zeros((nzz, n, n), np.float32)
    filled = C.c_double()
    stages = np.zeros(5, np.float64)
    _check(lib().ref_reconstruct(_p(f), C.c_int(count), C.c_int(n), _p(il), _p(_geom(geom)), C.c_int(nz),
                                 C.c_int(iterations), C.c_int(SOLVERS[solver]), C.c_int(TRANSFORMS[gp_transform]),
                                 C.c_float(tv_weight), C.c_int(tv_inner), _p(out), C.byref(filled), _p(stages)))
    if return_stages:
        return out, filled.value, dict(zip(["fft2", "mapping", "normalize", "solve", "finish"], stages))
    return out, filled.value


def tv_prox(b, dual_p, lam, inner):
    """cpu::tv_prox (src/cpu/tv.cpp:7-44) on a dense volume; dual_p (3, nz, ny, nx) is updated."""
    b = _f32(b)
    p = _f32(dual_p).copy()
    x = np.zeros_like(b)
    _check(lib().ref_tv_prox(_p(b), _p(x), _p(p), *map(C.c_int, b.shape), C.c_float(lam), C.c_int(inner)))
    return x, p


def bpm_tables(n, nz, illuminations, geom, obliquity=True):
    il = _illum(illuminations)
    count = il.shape[0]
    step = np.zeros((count, n, n), np.complex64)
    last = np.zeros((count, n, n), np.complex64)
    q = np.zeros((count, n, n), np.float32)
    pl = np.zeros(2, np.float32)
    _check(lib().ref_bpm_tables(C.c_int(n), C.c_int(nz), _p(il), C.c_int(count), _p(_geom(geom)),
                                C.c_int(int(obliquity)), _p(step), _p(last), _p(q), _p(pl)))
    return dict(step=step, last=last, q=q, phase=float(pl[0]), lipschitz=float(pl[1]))


def bpm_forward(ri, illuminations, geom, obliquity=True):
    ri = _f32(ri)
    il = _illum(illuminations)
    nz, n = ri.shape[0], ri.shape[2]
    out = np.zeros((il.shape[0], n, n), np.complex64)
    _check(lib().ref_bpm_forward(_p(ri), C.c_int(nz), C.c_int(n), _p(il), C.c_int(il.shape[0]), _p(_geom(geom)),
                                 C.c_int(int(obliquity)), _p(out)))
    return out


def bpm_vjp(x, r, illuminations, geom, obliquity=True):
    """cpu::bpm_vjp (src/cpu/bpm.cpp:178-189); x is the contrast n - n_medium."""
    x, r = _f32(x), _c64(r)
    il = _illum(illuminations)
    out = np.zeros_like(x)
    _check(lib().ref_bpm_vjp(_p(x), C.c_int(x.shape[0]), C.c_int(x.shape[2]), _p(r), _p(il), C.c_int(il.shape[0]),
                             _p(_geom(geom)), C.c_int(int(obliquity)), _p(out)))
    return out


def bpm_jvp(x, h, illuminations, geom, obliquity=True):
    x, h = _f32(x), _f32(h)
    il = _illum(illuminations)
    out = np.zeros((il.shape[0], x.shape[1], x.shape[2]), np.complex64)
    _check(lib().ref_bpm_jvp(_p(x), _p(h), C.c_int(x.shape[0]), C.c_int(x.shape[2]), _p(il), C.c_int(il.shape[0]),
                             _p(_geom(geom)), C.c_int(int(obliquity)), _p(out)))
    return out


def bpm_reconstruct(fields, illuminations, geom, initial, iterations=20, batch=0, step=1.0, tv_weight=0.0,
                    tv_inner=10, obliquity=True):
    f, init = _c64(fields), _f32(initial)
    il = _illum(illuminations)
    out = np.zeros_like(init)
    loss = np.zeros(max(iterations, 1), np.float64)
    _check(lib().ref_bpm_reconstruct(_p(f), C.c_int(f.shape[0]), C.c_int(f.shape[2]), _p(il), _p(_geom(geom)),
                                     _p(init), C.c_int(init.shape[0]), C.c_int(iterations), C.c_int(batch),
                                     C.c_float(step), C.c_float(tv_weight), C.c_int(tv_inner),
                                     C.c_int(int(obliquity)), _p(out), _p(loss)))
    return out, loss[:iterations]


def _spheres(spheres):
    return np.ascontiguousarray(np.reshape(spheres, (-1, 5)), np.float32)


def render_phantom(spheres, geom, nz, n):
    s = _spheres(spheres)
    out = np.zeros((nz, n, n), np.float32)
    _check(lib().ref_render_phantom(_p(s), C.c_int(s.shape[0]), _p(_geom(geom)), C.c_int(nz), C.c_int(n), _p(out)))
    return out


MODELS = {"born": 0, "rytov": 1, "exact": 2}


def forward_fields(spheres, illuminations, geom, n, model="rytov"):
    s = _spheres(spheres)
    il = _illum(illuminations)
    out = np.zeros((il.shape[0], n, n), np.complex64)
    _check(lib().ref_forward_fields(_p(s), C.c_int(s.shape[0]), _p(il), C.c_int(il.shape[0]), _p(_geom(geom)),
                                    C.c_int(n), C.c_int(MODELS[model]), _p(out)))
    return out


def synthesize_holograms(ratio, illuminations, geom, carrier=(5.0, 5.0), reference_amplitude=1.0, noise=0.0,
                         seed=1):
    r = _c64(ratio)
    il = _illum(illuminations)
    out = np.zeros(r.shape, np.float32)
    _check(lib().ref_synthesize_holograms(_p(r), *map(C.c_int, r.shape), _p(il), _p(_geom(geom)),
                                          C.c_float(carrier[0]), C.c_float(carrier[1]),
                                          C.c_float(reference_amplitude), C.c_float(noise),
                                          C.c_ulonglong(seed), _p(out)))
    return out


def pipeline(holo, bg, center, radius, output_size, illuminations, geom, nz=0, iterations=0, solver="gp",
             gp_transform="r2c", tv_weight=1e-2, tv_inner=10, runs=1):
    """The CPU Pipeline (src/pipeline.cpp:18-64): returns (ri, filled, ms) with ms the setup,
    set_background, run and stage times in milliseconds."""
    h, b = _f32(holo), _f32(bg)
    count, n = h.shape[0], h.shape[2]
    il = _illum(illuminations)
    m = output_size if output_size > 0 else n
    nzz = nz if nz > 0 else m
    out = np.zeros((nzz, m, m), np.float32)
    filled = C.c_double()
    ms = np.zeros(11, np.float64)
    _check(lib().ref_pipeline(_p(h), _p(b), C.c_int(count), C.c_int(n), C.c_float(center[0]), C.c_float(center[1]),
                              C.c_float(radius), C.c_int(output_size), _p(il), _p(_geom(geom)), C.c_int(nz),
                              C.c_int(iterations), C.c_int(SOLVERS[solver]), C.c_int(TRANSFORMS[gp_transform]),
                              C.c_float(tv_weight), C.c_int(tv_inner), C.c_int(runs), _p(out), C.byref(filled),
                              _p(ms)))
    names = ["setup", "set_background", "run", "fields", "rytov", "fft2", "mapping", "normalize", "solve",
             "finish", "total"]
    return out, filled.value, dict(zip(names, ms))


def pipeline_errors(count, n, illuminations, geom):
    il = _illum(illuminations)
    codes = np.zeros(2, np.int32)
    lib().ref_pipeline_errors(C.c_int(count), C.c_int(n), _p(il), _p(_geom(geom)), _p(codes))
    return int(codes[0]), int(codes[1])


def ewald_half(spectra, illuminations, geom, nz=0):
    """The reference's Ewald mapping and Hermitian half data (ref_ewald_half) on spectra (count, n, n)
    complex64: returns (a (nz, n, n/2+1) complex64, hits uint8, filled voxel count)."""
    s = _c64(spectra)
    count, n = s.shape[0], s.shape[2]
    nzz = nz if nz > 0 else n
    il = _illum(illuminations)
    a = np.zeros((nzz, n, n // 2 + 1), np.complex64)
    hits = np.zeros(a.shape, np.uint8)
    filled = C.c_longlong()
    _check(lib().ref_ewald_half(_p(s), C.c_int(count), C.c_int(n), C.c_int(nzz), _p(il), _p(_geom(geom)), _p(a),
                                _p(hits), C.byref(filled)))
    return a, hits, int(filled.value)
