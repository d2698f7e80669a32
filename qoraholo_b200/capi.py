"""ctypes binding of the C ABI in include/qoraholo_b200.h (libqhk.so).

This is the device-level interface: plans and kernels take device pointers (ints; e.g. a torch
tensor's ``data_ptr()``) and a CUDA stream handle. The reference-compatible numpy API lives in
``qoraholo_b200`` (``__init__.py``) on top of the C++ host layer. Loading fails loudly if the
library has not been built (``python qoraholo_b200/_build.py``); there is no fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

# QHK_LIBRARY selects another build of the same ABI, e.g. the debug build qoraholo_b200/debug/libqhk.so.
LIB_PATH = Path(os.environ.get("QHK_LIBRARY") or Path(__file__).resolve().parent / "libqhk.so")

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


class RequestTimes(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("service_ms", C.c_double), ("total_ms", C.c_double),
                ("gpu_ms", C.c_double)]


class ServerCounters(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64), ("cancelled", C.c_uint64),
                ("workspaces_created", C.c_uint64), ("workspaces_evicted", C.c_uint64),
                ("graph_launches", C.c_uint64), ("passed_over", C.c_uint64), ("budget", C.c_size_t),
                ("used", C.c_size_t), ("peak_used", C.c_size_t), ("geometries", C.c_int), ("inflight", C.c_int),
                ("peak_inflight", C.c_int)]


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
    "qhk_wait_timeouts": (_I, [C.POINTER(C.c_uint64)]),
    "qhk_debug_enabled": (_I, []),
    "qhk_debug_violations": (_I, [C.POINTER(C.c_uint64), _I]),
    "qhk_pinned_alloc": (_I, [C.c_size_t, C.POINTER(_VP)]),
    "qhk_pinned_free": (_I, [_VP]),
    "qhk_tv_prox_workspace": (_I, [_VP, _VP, _VP, _I, _I, _I, _I, _F, _I, _VP]),
    "qhk_unwrap_noalloc": (_I, [_VP, _VP, _I, _I, _I, _VP]),
    "qhk_bpm_vjp": (_I, [_VP, _I, _I, _VP, _VP, _I, C.POINTER(Geometry), _I, _VP]),
    "qhk_pipeline_create": (_I, [C.POINTER(_VP), _VP, _VP, C.POINTER(Geometry)]),
    "qhk_pipeline_set_background": (_I, [_VP, _VP]),
    "qhk_pipeline_input": (_VP, [_VP]),
    "qhk_pipeline_output": (_VP, [_VP]),
    "qhk_pipeline_process": (_I, [_VP]),
    "qhk_pipeline_run": (_I, [_VP, _VP, _VP]),
    "qhk_pipeline_run_stream": (_I, [_VP, _VP, C.c_int, _VP]),
    "qhk_pipeline_process_device": (_I, [_VP, _VP, _VP, _VP]),
    "qhk_pipeline_result": (_I, [_VP, C.POINTER(C.c_double), _VP]),
    "qhk_pipeline_filled": (_I, [_VP, _VP, C.POINTER(C.c_double)]),
    "qhk_pipeline_check_waits": (_I, [_VP, _VP]),
    "qhk_pipeline_wait_probe": (_I, [_VP, _I]),
    "qhk_pipeline_time_prox": (_I, [_VP, _I]),
    "qhk_pipeline_prox_time": (_I, [_VP, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "qhk_pipeline_shape": (_I, [_VP, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    "qhk_pipeline_device_bytes": (C.c_size_t, [_VP]),
    "qhk_pipeline_destroy": (_I, [_VP]),
    "qhk_pipeline_create_batched": (_I, [C.POINTER(_VP), _VP, _VP, C.POINTER(Geometry), _I]),
    "qhk_pipeline_process_device_graph": (_I, [_VP, _VP, _VP, _VP]),
    "qhk_pipeline_filled_batch": (_I, [_VP, _VP, _VP]),
    "qhk_unwrap_batch_create": (_I, [C.POINTER(_VP), _VP, _VP, _I]),
    "qhk_unwrap_batch_offset": (C.c_size_t, [_VP, _I]),
    "qhk_unwrap_batch_total": (C.c_size_t, [_VP]),
    "qhk_unwrap_batch_run": (_I, [_VP, _VP, _VP, _I, _VP]),
    "qhk_unwrap_batch_device_bytes": (C.c_size_t, [_VP]),
    "qhk_unwrap_batch_destroy": (_I, [_VP]),
    "qhk_synthesize_holograms_device": (_I, [_VP, _I, _I, _VP, C.c_double, C.c_double, C.c_double, C.c_double, _F,
                                             C.c_uint64, _VP, _VP]),
    "qhk_autotune_enable": (_I, [_I]),
    "qhk_autotune_radix": (_I, [_I]),
    "qhk_fft_axis_engine": (_I, [_I]),
    "qhk_selftest_rcp_sqrt": (_I, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "qhk_tv_form": (_I, [_I]),
    "qhk_autotune_report": (C.c_size_t, [_VP, C.c_size_t]),
    "qhk_server_create": (_I, [C.POINTER(_VP), C.c_size_t, _I, _I]),
    "qhk_server_add_geometry": (_I, [_VP, _VP, _VP, C.POINTER(Geometry), _VP, C.POINTER(_I)]),
    "qhk_server_remove_geometry": (_I, [_VP, _I]),
    "qhk_server_volume_shape": (_I, [_VP, _I, C.POINTER(_I), C.POINTER(_I)]),
    "qhk_server_submit": (_I, [_VP, _I, _VP, _VP, C.POINTER(C.c_uint64)]),
    "qhk_server_done": (_I, [_VP, C.c_uint64, C.POINTER(_I)]),
    "qhk_server_wait": (_I, [_VP, C.c_uint64, C.POINTER(C.c_double), C.POINTER(RequestTimes)]),
    "qhk_server_cancel": (_I, [_VP, C.c_uint64, C.POINTER(_I)]),
    "qhk_server_stats": (_I, [_VP, C.POINTER(ServerCounters)]),
    "qhk_server_destroy": (_I, [_VP]),
    "qhk_admission_simulate": (_I, [C.c_size_t, _I, _I, _I, _VP, _VP, _VP, _I, _VP, _VP, _VP, C.POINTER(_I)]),
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


def tv_prox_workspace(d_b, d_x, d_work, work_volumes, nz, ny, nx, lam, inner, stream=0):
    """No-allocation proximal step on a caller workspace of 9 or 12 volumes (the dual first); with 12
    the two-step FGP form can run."""
    check(lib().qhk_tv_prox_workspace(_VP(d_b), _VP(d_x), _VP(d_work), int(work_volumes), nz, ny, nx, float(lam),
                                      int(inner), _VP(stream)))


def unwrap_noalloc(d_wrapped, d_unwrapped, count, ny, nx, stream=0):
    """qhk_unwrap_noalloc: device in / device out, no allocation (scratch in a static device array)."""
    check(lib().qhk_unwrap_noalloc(_VP(d_wrapped), _VP(d_unwrapped), count, ny, nx, _VP(stream)))


def pinned_array(shape, dtype=np.float32) -> np.ndarray:
    """A numpy array in page-locked host memory (qhk_pinned_alloc), freed when the array is released:
    qhk_pipeline_run transfers such buffers directly, without staging copies."""
    import weakref

    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    ptr = _VP()
    check(lib().qhk_pinned_alloc(nbytes, C.byref(ptr)))
    raw = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(nbytes,))
    arr = raw.view(dtype).reshape(shape)
    weakref.finalize(arr, lib().qhk_pinned_free, _VP(ptr.value))
    return arr


def wait_timeouts() -> int:
    """Bounded device waits that ran out since the library was loaded (qhk_wait_timeouts); 0 in every
    correct run."""
    n = C.c_uint64()
    check(lib().qhk_wait_timeouts(C.byref(n)))
    return n.value


def debug_enabled() -> bool:
    """True when the loaded library is the debug build (device bounds checks compiled in)."""
    return bool(lib().qhk_debug_enabled())


def debug_violations(reset: bool = False) -> tuple[int, str]:
    """Failed device bounds checks of the debug build since the last reset, and where the first one
    was (qhk_debug_violations); (0, "") in the release build."""
    n = C.c_uint64()
    check(lib().qhk_debug_violations(C.byref(n), int(bool(reset))))
    where = lib().qhk_last_error().decode() if n.value else ""
    return n.value, where


def autotune_enable(enabled: bool = True):
    """Plans built from now on time their launch shapes (on by default)."""
    check(lib().qhk_autotune_enable(int(bool(enabled))))


def autotune_radix(enabled: bool = True):
    """Plans built from now on also time the FFT decomposition of their axis passes (off by default: the
    variants round differently, so results then depend on which one won)."""
    check(lib().qhk_autotune_radix(int(bool(enabled))))


def fft_axis_engine(engine: int = -1):
    """Force the FFT decomposition of the register-covered axis passes (0 staged, 1 or 2 register
    variants; -1 tuned / default). For tests and comparisons."""
    check(lib().qhk_fft_axis_engine(int(engine)))


def selftest_rcp_sqrt():
    """(mismatches, first mismatching input bits) of the projection factor against the IEEE operations
    over every float in [1, 2^126) (qhk_selftest_rcp_sqrt)."""
    n, b = C.c_uint64(), C.c_uint32()
    check(lib().qhk_selftest_rcp_sqrt(C.byref(n), C.byref(b)))
    return n.value, b.value


def synthesize_holograms_device(d_ratio, count, n, illuminations, pixel, carrier=(5.0, 5.0), reference_amplitude=1.0,
                                noise=0.0, seed=1, d_out=0, stream=0):
    """Off-axis holograms on the device from device field ratios (count, n, n) complex64 into d_out
    (count, n, n) float32 (qhk_synthesize_holograms_device)."""
    il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
    check(lib().qhk_synthesize_holograms_device(_VP(d_ratio), int(count), int(n), host_ptr(il), float(pixel),
                                                float(carrier[0]), float(carrier[1]), float(reference_amplitude),
                                                float(noise), int(seed) & ((1 << 64) - 1), _VP(d_out), _VP(stream)))


def tv_form(form: int):
    """FGP step form: 0 tuned (default), 1 stored extrapolated point, 2 recomputed (same results)."""
    check(lib().qhk_tv_form(int(form)))


def autotune_report() -> str:
    """The tuned launch shapes so far, one line per (family, shape)."""
    n = lib().qhk_autotune_report(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().qhk_autotune_report(C.cast(buf, _VP), n + 1)
    return buf.value.decode()


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


class UnwrapBatch:
    """qhk_unwrap_batch_*: least-squares unwrap of images of uneven sizes packed in one device buffer,
    one persistent launch per pass for the whole batch. `shapes`: (ny, nx) per image; `offsets[i]`
    is the first float of image i; `total` the packed length."""

    def __init__(self, shapes):
        sh = np.ascontiguousarray(np.reshape(shapes, (-1, 2)), np.int32)
        ny = np.ascontiguousarray(sh[:, 0])
        nx = np.ascontiguousarray(sh[:, 1])
        self._h = _VP()
        check(lib().qhk_unwrap_batch_create(C.byref(self._h), host_ptr(ny), host_ptr(nx), len(sh)))
        self.shapes = [tuple(map(int, r)) for r in sh]
        self.offsets = [int(lib().qhk_unwrap_batch_offset(self._h, i)) for i in range(len(sh))]
        self.total = int(lib().qhk_unwrap_batch_total(self._h))

    def run(self, d_wrapped, d_unwrapped, stream=0, graph=False):
        check(lib().qhk_unwrap_batch_run(self._h, _VP(d_wrapped), _VP(d_unwrapped), int(bool(graph)), _VP(stream)))

    @property
    def device_bytes(self):
        return int(lib().qhk_unwrap_batch_device_bytes(self._h))

    def pack(self, images):
        """Host images (a list of (ny, nx) float32 arrays) -> one packed float32 array."""
        return np.concatenate([np.ascontiguousarray(a, np.float32).ravel() for a in images])

    def unpack(self, packed):
        return [packed[o:o + ny * nx].reshape(ny, nx) for o, (ny, nx) in zip(self.offsets, self.shapes)]

    def close(self):
        if self._h:
            check(lib().qhk_unwrap_batch_destroy(self._h))
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pipeline:
    """qhk_pipeline_*: holograms -> index with resident device state. `process()` works from the
    page-locked input buffer (``input`` view); `process_device` from device pointers. With
    ``batch`` > 1, `batch` requests of this geometry run together (one launch per pass): input
    (batch * count, N, N), output (batch, nz, n, n)."""

    def __init__(self, count, hologram_size, center, illuminations, geom, radius=0.0, output_size=0, upload_chunks=1,
                 batch=1, **odt):
        self._il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
        o = PipelineOptions(int(count), int(hologram_size), float(center[0]), float(center[1]), float(radius),
                            int(output_size), int(upload_chunks), odt_options(**odt))
        self._h = _VP()
        self.batch = int(batch)
        if self.batch == 1:
            check(lib().qhk_pipeline_create(C.byref(self._h), C.byref(o), host_ptr(self._il),
                                            C.byref(geometry(geom))))
        else:
            check(lib().qhk_pipeline_create_batched(C.byref(self._h), C.byref(o), host_ptr(self._il),
                                                    C.byref(geometry(geom)), self.batch))
        nz, ny, nx = _I(), _I(), _I()
        check(lib().qhk_pipeline_shape(self._h, C.byref(nz), C.byref(ny), C.byref(nx)))
        self.shape = (nz.value, ny.value, nx.value) if self.batch == 1 else (self.batch, nz.value, ny.value, nx.value)
        self.input_shape = (int(count) * self.batch, int(hologram_size), int(hologram_size))
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

    def run(self, holograms, out=None):
        """qhk_pipeline_run: host holograms (input_shape) -> a new (or the given) host volume array."""
        h = np.ascontiguousarray(holograms, np.float32)
        if h.shape != self.input_shape:
            raise ValueError(f"holograms must have shape {self.input_shape}")
        if out is None:
            out = np.empty(self.shape, np.float32)
        elif out.shape != self.shape or out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {self.shape}")
        check(lib().qhk_pipeline_run(self._h, host_ptr(h), host_ptr(out)))
        return out

    def run_stream(self, holograms, out=None):
        """qhk_pipeline_run_stream: host holograms (items, *input_shape) -> (items, *shape), the
        transfers of each stack overlapping the solve of the next."""
        h = np.ascontiguousarray(holograms, np.float32)
        if h.ndim != 1 + len(self.input_shape) or h.shape[1:] != self.input_shape or h.shape[0] < 1:
            raise ValueError(f"holograms must have shape (items, {', '.join(map(str, self.input_shape))})")
        shape = (h.shape[0],) + tuple(self.shape)
        if out is None:
            out = np.empty(shape, np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {shape}")
        check(lib().qhk_pipeline_run_stream(self._h, host_ptr(h), int(h.shape[0]), host_ptr(out)))
        return out

    def process_device(self, d_holo, d_index, stream=0):
        check(lib().qhk_pipeline_process_device(self._h, _VP(d_holo), _VP(d_index), _VP(stream)))

    def process_device_graph(self, d_holo, d_index, stream=0):
        """process_device replayed as one CUDA graph (the first call for these buffers runs directly)."""
        check(lib().qhk_pipeline_process_device_graph(self._h, _VP(d_holo), _VP(d_index), _VP(stream)))

    def filled_batch(self, stream=0):
        out = np.zeros(self.batch, np.float64)
        check(lib().qhk_pipeline_filled_batch(self._h, _VP(stream), host_ptr(out)))
        return out

    def result(self):
        filled = C.c_double()
        t = PipelineTimings()
        check(lib().qhk_pipeline_result(self._h, C.byref(filled), C.cast(C.pointer(t), _VP)))
        return filled.value, {name: getattr(t, name) for name in TIMING_NAMES}

    def filled_device(self, stream=0):
        v = C.c_double()
        check(lib().qhk_pipeline_filled(self._h, _VP(stream), C.byref(v)))
        return v.value

    def check_waits(self, stream=0):
        """Waits for `stream`; raises QhkError (TIMEOUT) if a bounded device wait of this pipeline ran
        out since the last check (device-form runs cannot report it themselves)."""
        check(lib().qhk_pipeline_check_waits(self._h, _VP(stream)))

    def time_prox(self, enable=True):
        """Record CUDA events around the TV proximal steps of the following direct runs
        (qhk_pipeline_time_prox)."""
        check(lib().qhk_pipeline_time_prox(self._h, int(bool(enable))))

    def prox_time(self):
        """(milliseconds, FGP launches) of the proximal steps recorded since time_prox or the last call."""
        ms, n = C.c_double(), C.c_uint64()
        check(lib().qhk_pipeline_prox_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def wait_probe(self, polls=1000):
        """Test hook of the timeout path: one bounded wait that nothing completes, counted in this
        pipeline's counter; raises QhkError (TIMEOUT) as a run whose wait ran out does."""
        check(lib().qhk_pipeline_wait_probe(self._h, int(polls)))

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


class Server:
    """qhk_server_*: the serving loop. Register geometries (resident background fields and plans),
    then submit hologram stacks from any thread and wait for their index volumes. Requests are
    admitted as execution slots and device memory (``hbm_budget`` bytes) free up, and run
    concurrently on the GPU; each result is the same as that request run alone."""

    def __init__(self, hbm_budget=40 << 30, max_inflight=4, use_graphs=True):
        self._h = _VP()
        check(lib().qhk_server_create(C.byref(self._h), int(hbm_budget), int(max_inflight), int(bool(use_graphs))))
        self._shapes = {}
        self._inputs = {}
        self._live = {}

    def add_geometry(self, count, hologram_size, center, illuminations, geom, backgrounds, radius=0.0,
                     output_size=0, **odt):
        """Registers a geometry (validated like Pipeline) with its background holograms
        (count, N, N); returns its id."""
        il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
        o = PipelineOptions(int(count), int(hologram_size), float(center[0]), float(center[1]), float(radius),
                            int(output_size), 1, odt_options(**odt))
        bg = np.ascontiguousarray(backgrounds, np.float32)
        if bg.shape != (int(count), int(hologram_size), int(hologram_size)):
            raise ValueError("Server: backgrounds must be (count, N, N)")
        gid = _I()
        check(lib().qhk_server_add_geometry(self._h, C.byref(o), host_ptr(il), C.byref(geometry(geom)), host_ptr(bg),
                                            C.byref(gid)))
        nz, n = _I(), _I()
        check(lib().qhk_server_volume_shape(self._h, gid.value, C.byref(nz), C.byref(n)))
        self._shapes[gid.value] = ((int(count), int(hologram_size), int(hologram_size)), (nz.value, n.value, n.value))
        return gid.value

    def remove_geometry(self, gid):
        check(lib().qhk_server_remove_geometry(self._h, int(gid)))
        self._shapes.pop(int(gid), None)

    def volume_shape(self, gid):
        return self._shapes[int(gid)][1]

    def submit(self, gid, holograms, out=None):
        """Queues one stack (count, N, N) float32; returns a ticket. `out` (optional) is a float32
        array of the volume's shape to write into; both arrays are kept alive until wait()."""
        in_shape, vol_shape = self._shapes[int(gid)]
        h = np.ascontiguousarray(holograms, np.float32)
        if h.shape != in_shape:
            raise ValueError(f"Server: holograms must be {in_shape}")
        if out is None:
            out = np.empty(vol_shape, np.float32)
        elif out.shape != vol_shape or out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"Server: out must be a C-contiguous float32 array of shape {vol_shape}")
        t = C.c_uint64()
        check(lib().qhk_server_submit(self._h, int(gid), host_ptr(h), host_ptr(out), C.byref(t)))
        self._live[t.value] = (h, out)
        return t.value

    def done(self, ticket):
        d = _I()
        check(lib().qhk_server_done(self._h, int(ticket), C.byref(d)))
        return bool(d.value)

    def cancel(self, ticket):
        """Withdraws a request that has not started; True if it was withdrawn (its wait() then raises)."""
        c = _I()
        check(lib().qhk_server_cancel(self._h, int(ticket), C.byref(c)))
        return bool(c.value)

    def wait(self, ticket):
        """Blocks until the request is done: (index volume, filled fraction, timings dict in ms)."""
        filled = C.c_double()
        t = RequestTimes()
        try:
            check(lib().qhk_server_wait(self._h, int(ticket), C.byref(filled), C.byref(t)))
        finally:
            arrays = self._live.pop(int(ticket), None)
        times = {"queue": t.queue_ms, "service": t.service_ms, "total": t.total_ms, "gpu": t.gpu_ms}
        return arrays[1], filled.value, times

    def stats(self):
        c = ServerCounters()
        check(lib().qhk_server_stats(self._h, C.byref(c)))
        return {name: getattr(c, name) for name, _ in ServerCounters._fields_}

    def close(self):
        if self._h:
            check(lib().qhk_server_destroy(self._h))
            self._h = _VP()
        self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def admission_simulate(budget, max_inflight, max_pass, resident, workspace, ops):
    """The serving loop's admission policy on the host alone (no device work): returns a list of
    (submission index, action, bytes in use) per admission, action 0 reuse, 1 allocate, 2 allocate
    after evicting idle workspaces. ops: geometry id to submit, or -1 to complete the oldest
    running request."""
    res = np.ascontiguousarray(resident, np.uint64)
    ws = np.ascontiguousarray(workspace, np.uint64)
    o = np.ascontiguousarray(ops, np.int32)
    n = max(len(o), 1)
    admitted = np.zeros(n, np.int32)
    action = np.zeros(n, np.int32)
    used = np.zeros(n, np.uint64)
    count = _I()
    check(lib().qhk_admission_simulate(int(budget), int(max_inflight), int(max_pass), len(res), host_ptr(res),
                                       host_ptr(ws), host_ptr(o), len(o), host_ptr(admitted), host_ptr(action),
                                       host_ptr(used), C.byref(count)))
    k = count.value
    return [(int(admitted[i]), int(action[i]), int(used[i])) for i in range(k)]
