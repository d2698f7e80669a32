"""ctypes binding of the C ABI in include/qoraholo_b200.h (libqhk.so).

This is the device-level interface: plans and kernels take device pointers (ints; e.g. a torch
tensor's ``data_ptr()``) and a CUDA stream handle. The reference-compatible numpy API lives in
``qoraholo_b200`` (``__init__.py``) on top of the C++ host layer. Loading fails loudly if the
library has not been built (``python qoraholo_b200/_build.py``); there is no fallback.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libqhk.so"

OK, INVALID_ARGUMENT, CUDA_ERROR, LOGIC_ERROR, OUT_OF_MEMORY, TIMEOUT, INTERNAL = range(7)
SOLVERS = {"gp": 0, "tv": 1}
TRANSFORMS = {"r2c": 0, "c2c": 1}
MAPPINGS = {"gather": 0, "scatter": 1}

_lib = None


class QhkError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class Geometry(C.Structure):
    _fields_ = [("wavelength", C.c_float), ("n_medium", C.c_float), ("na", C.c_float), ("pixel", C.c_float)]


class OdtOptions(C.Structure):
    _fields_ = [("nz", C.c_int), ("iterations", C.c_int), ("solver", C.c_int), ("gp_transform", C.c_int),
                ("tv_weight", C.c_float), ("tv_inner", C.c_int), ("mapping", C.c_int)]


class PipelineOptions(C.Structure):
    _fields_ = [("count", C.c_int), ("hologram_size", C.c_int), ("center_y", C.c_float), ("center_x", C.c_float),
                ("radius", C.c_float), ("output_size", C.c_int), ("upload_chunks", C.c_int), ("odt", OdtOptions)]


TIMING_NAMES = ["upload", "fields", "rytov", "fft2", "clear", "mapping", "normalize", "solve", "finish", "download",
                "total"]


class PipelineTimings(C.Structure):
    _fields_ = [(name, C.c_double) for name in TIMING_NAMES]


_VP = C.c_void_p
_I = C.c_int
_F = C.c_float
_PROTOS = {
    "qhk_last_error": (C.c_char_p, []),
    "qhk_device_present": (_I, []),
    "qhk_odt_create": (_I, [C.POINTER(_VP), _I, _I, _VP, C.POINTER(Geometry), C.POINTER(OdtOptions)]),
    "qhk_odt_run": (_I, [_VP, _VP, _VP, _VP]),
    "qhk_odt_filled": (_I, [_VP, _VP, C.POINTER(C.c_double)]),
    "qhk_odt_shape": (_I, [_VP, C.POINTER(_I), C.POINTER(_I)]),
    "qhk_odt_device_bytes": (C.c_size_t, [_VP]),
    "qhk_odt_destroy": (_I, [_VP]),
    "qhk_reconstruct": (_I, [_VP, _I, _I, _VP, C.POINTER(Geometry), C.POINTER(OdtOptions), _VP,
                             C.POINTER(C.c_double)]),
    "qhk_ewald_map": (_I, [_VP, _I, _I, _I, _VP, C.POINTER(Geometry), _I, _VP, _VP, _VP, _VP]),
    "qhk_tv_prox": (_I, [_VP, _VP, _VP, _I, _I, _I, _F, _I, _VP]),
    "qhk_fft2d": (_I, [_VP, _I, _I, _I, _F, _VP]),
    "qhk_rfft3": (_I, [_VP, _VP, _I, _I, _I, _VP]),
    "qhk_irfft3": (_I, [_VP, _VP, _I, _I, _I, _F, _VP]),
    "qhk_tv_prox_device": (_I, [_VP, _VP, _VP, _I, _I, _I, _F, _I, _VP]),
    "qhk_kernel_launches": (C.c_uint64, []),
    "qhk_unwrap_noalloc": (_I, [_VP, _VP, _I, _I, _I, _VP]),
    "qhk_bpm_vjp": (_I, [_VP, _I, _I, _VP, _VP, _I, C.POINTER(Geometry), _I, _VP]),
    "qhk_pipeline_create": (_I, [C.POINTER(_VP), _VP, _VP, C.POINTER(Geometry)]),
    "qhk_pipeline_set_background": (_I, [_VP, _VP]),
    "qhk_pipeline_input": (_VP, [_VP]),
    "qhk_pipeline_output": (_VP, [_VP]),
    "qhk_pipeline_process": (_I, [_VP]),
    "qhk_pipeline_process_device": (_I, [_VP, _VP, _VP, _VP]),
    "qhk_pipeline_result": (_I, [_VP, C.POINTER(C.c_double), _VP]),
    "qhk_pipeline_filled": (_I, [_VP, _VP, C.POINTER(C.c_double)]),
    "qhk_pipeline_shape": (_I, [_VP, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    "qhk_pipeline_device_bytes": (C.c_size_t, [_VP]),
    "qhk_pipeline_destroy": (_I, [_VP]),
}


def lib():
    """The loaded libqhk.so with argument types declared."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python qoraholo_b200/_build.py`")
        _lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _PROTOS.items():
            f = getattr(_lib, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
    return _lib


def check(code):
    if code != OK:
        msg = lib().qhk_last_error().decode()
        if code == INVALID_ARGUMENT:
            raise ValueError(msg)
        raise QhkError(code, msg)


def geometry(g) -> Geometry:
    w, nm, na, px = (float(v) for v in (g if not hasattr(g, "wavelength") else (g.wavelength, g.n_medium, g.na, g.pixel)))
    return Geometry(w, nm, na, px)


def odt_options(nz=0, iterations=0, solver="gp", gp_transform="r2c", tv_weight=1e-2, tv_inner=10,
                mapping="gather") -> OdtOptions:
    return OdtOptions(int(nz), int(iterations), SOLVERS[solver], TRANSFORMS[gp_transform], float(tv_weight),
                      int(tv_inner), MAPPINGS[mapping])


def host_ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_VP)


def device_present() -> bool:
    return bool(lib().qhk_device_present())


class OdtPlan:
    """Device-resident solver for one geometry (qhk_odt_*): fields -> index, no allocation per run."""

    def __init__(self, n, count, illuminations, geom, **options):
        self._il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
        self._h = _VP()
        check(lib().qhk_odt_create(C.byref(self._h), int(n), int(count), host_ptr(self._il), C.byref(geometry(geom)),
                                   C.byref(odt_options(**options))))
        nz, nn = _I(), _I()
        check(lib().qhk_odt_shape(self._h, C.byref(nz), C.byref(nn)))
        self.shape = (nz.value, nn.value, nn.value)

    def run(self, d_fields: int, d_index: int, stream: int = 0):
        check(lib().qhk_odt_run(self._h, _VP(d_fields), _VP(d_index), _VP(stream)))

    def filled(self, stream: int = 0) -> float:
        v = C.c_double()
        check(lib().qhk_odt_filled(self._h, _VP(stream), C.byref(v)))
        return v.value

    @property
    def device_bytes(self) -> int:
        return int(lib().qhk_odt_device_bytes(self._h))

    def close(self):
        if self._h:
            check(lib().qhk_odt_destroy(self._h))
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reconstruct(fields, illuminations, geom, **options):
    """qhk_reconstruct: host complex64 fields (count, n, n) -> (ri, filled)."""
    f = np.ascontiguousarray(fields, np.complex64)
    il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
    count, n = f.shape[0], f.shape[2]
    nz = options.get("nz", 0) or n
    out = np.zeros((nz, n, n), np.float32)
    filled = C.c_double()
    check(lib().qhk_reconstruct(host_ptr(f), count, n, host_ptr(il), C.byref(geometry(geom)),
                                C.byref(odt_options(**options)), host_ptr(out), C.byref(filled)))
    return out, filled.value


def ewald_map(d_spectra, count, n, nz, illuminations, geom, half, d_data, d_hits, d_filled, stream=0):
    il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
    check(lib().qhk_ewald_map(_VP(d_spectra), count, n, nz, host_ptr(il), C.byref(geometry(geom)), int(half),
                              _VP(d_data), _VP(d_hits), _VP(d_filled), _VP(stream)))


def tv_prox(d_b, d_x, d_dual, nz, ny, nx, lam, inner, stream=0):
    check(lib().qhk_tv_prox(_VP(d_b), _VP(d_x), _VP(d_dual), nz, ny, nx, float(lam), int(inner), _VP(stream)))


def tv_prox_device(d_b, d_x, d_dual9, nz, ny, nx, lam, inner, stream=0):
    """No-allocation proximal step: d_dual9 holds the dual (3 volumes) and 6 volumes of scratch."""
    check(lib().qhk_tv_prox_device(_VP(d_b), _VP(d_x), _VP(d_dual9), nz, ny, nx, float(lam), int(inner), _VP(stream)))


def unwrap_noalloc(d_wrapped, d_unwrapped, count, ny, nx, stream=0):
    """qhk_unwrap_noalloc: device in / device out, no allocation (scratch in a static device array)."""
    check(lib().qhk_unwrap_noalloc(_VP(d_wrapped), _VP(d_unwrapped), count, ny, nx, _VP(stream)))


def kernel_launches() -> int:
    return int(lib().qhk_kernel_launches())


def fft2d(d_data, count, n, forward=True, scale=1.0, stream=0):
    check(lib().qhk_fft2d(_VP(d_data), count, n, int(forward), float(scale), _VP(stream)))


def rfft3(d_x, d_half, nz, ny, nx, stream=0):
    check(lib().qhk_rfft3(_VP(d_x), _VP(d_half), nz, ny, nx, _VP(stream)))


def irfft3(d_half, d_x, nz, ny, nx, scale=1.0, stream=0):
    check(lib().qhk_irfft3(_VP(d_half), _VP(d_x), nz, ny, nx, float(scale), _VP(stream)))


def bpm_vjp(x, r, illuminations, geom, obliquity=True):
    """qhk_bpm_vjp: J^T r for the contrast x (host arrays)."""
    x = np.ascontiguousarray(x, np.float32)
    r = np.ascontiguousarray(r, np.complex64)
    il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
    out = np.zeros_like(x)
    check(lib().qhk_bpm_vjp(host_ptr(x), x.shape[0], x.shape[2], host_ptr(r), host_ptr(il), il.shape[0],
                            C.byref(geometry(geom)), int(obliquity), host_ptr(out)))
    return out


class Pipeline:
    """qhk_pipeline_*: holograms -> index with resident device state. `process()` works from the
    page-locked input buffer (``input`` view); `process_device` from device pointers."""

    def __init__(self, count, hologram_size, center, illuminations, geom, radius=0.0, output_size=0, upload_chunks=1,
                 **odt):
        self._il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
        o = PipelineOptions(int(count), int(hologram_size), float(center[0]), float(center[1]), float(radius),
                            int(output_size), int(upload_chunks), odt_options(**odt))
        self._h = _VP()
        check(lib().qhk_pipeline_create(C.byref(self._h), C.byref(o), host_ptr(self._il), C.byref(geometry(geom))))
        nz, ny, nx = _I(), _I(), _I()
        check(lib().qhk_pipeline_shape(self._h, C.byref(nz), C.byref(ny), C.byref(nx)))
        self.shape = (nz.value, ny.value, nx.value)
        self.input_shape = (int(count), int(hologram_size), int(hologram_size))
        n_in = int(np.prod(self.input_shape))
        n_out = int(np.prod(self.shape))
        self.input = np.ctypeslib.as_array(C.cast(lib().qhk_pipeline_input(self._h), C.POINTER(C.c_float)),
                                           shape=(n_in,)).reshape(self.input_shape)
        self.output = np.ctypeslib.as_array(C.cast(lib().qhk_pipeline_output(self._h), C.POINTER(C.c_float)),
                                            shape=(n_out,)).reshape(self.shape)

    def set_background(self, backgrounds):
        b = np.ascontiguousarray(backgrounds, np.float32)
        check(lib().qhk_pipeline_set_background(self._h, host_ptr(b)))

    def process(self):
        check(lib().qhk_pipeline_process(self._h))

    def process_device(self, d_holo, d_index, stream=0):
        check(lib().qhk_pipeline_process_device(self._h, _VP(d_holo), _VP(d_index), _VP(stream)))

    def result(self):
        filled = C.c_double()
        t = PipelineTimings()
        check(lib().qhk_pipeline_result(self._h, C.byref(filled), C.cast(C.pointer(t), _VP)))
        return filled.value, {name: getattr(t, name) for name in TIMING_NAMES}

    def filled_device(self, stream=0):
        v = C.c_double()
        check(lib().qhk_pipeline_filled(self._h, _VP(stream), C.byref(v)))
        return v.value

    @property
    def device_bytes(self):
        return int(lib().qhk_pipeline_device_bytes(self._h))

    def close(self):
        """Releases the pipeline; the `input` / `output` views become invalid."""
        self.input = self.output = None
        if self._h:
            check(lib().qhk_pipeline_destroy(self._h))
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
