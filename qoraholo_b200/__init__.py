"""Optical diffraction tomography -- holograms to refractive index -- on NVIDIA B200.

A drop-in for the ``qoraholo`` Python package: every public name, argument, default and return form
follows python/qoraholo/__init__.py of QoraHolo, and the work runs in this project's sm_100a kernels
behind the C ABI of ``libqhk.so`` (include/qoraholo_b200.h). ``backend`` is accepted everywhere and
defaults to ``"cuda"``; this build has no host implementation, so ``"cpu"`` raises.

Conventions: numpy arrays; images square with an even side and their origin at pixel n/2; image
functions take one image (2D) or a stack (count, n, n) and answer with the rank they were given;
lengths in micrometres, spatial frequencies in cycles per micrometre; illuminations as (count, 2)
pairs (fy, fx).
"""

from __future__ import annotations

import numpy as np

try:
    from . import _core  # noqa: E402
except ImportError as e:  # no fallback: without the native libraries nothing here can run
    raise ImportError(
        "qoraholo_b200 native extension is not built; run `python qoraholo_b200/_build.py`"
    ) from e

from ._core import Geometry, Sideband, Sphere, cuda_available  # noqa: E402

__all__ = [
    "Geometry",
    "Pipeline",
    "Sideband",
    "Sphere",
    "bpm_forward",
    "bpm_reconstruct",
    "circular_scan",
    "cuda_available",
    "extract_fields",
    "field_ratio",
    "find_sideband",
    "forward_fields",
    "reconstruct",
    "render_phantom",
    "rytov",
    "synthesize_holograms",
    "unwrap",
]


class _Images:
    """A C-contiguous 3D stack of `dtype` made from an image or a stack, remembering which it was,
    so that results go back in the caller's rank."""

    def __init__(self, a, dtype):
        arr = np.ascontiguousarray(a, dtype=dtype)
        if arr.ndim not in (2, 3):
            raise ValueError(f"expected a 2D image or a 3D stack, got {arr.ndim} dimensions")
        self.was_image = arr.ndim == 2
        self.stack = arr[np.newaxis] if self.was_image else arr

    def give_back(self, result):
        return result[0] if self.was_image else result


def _views(illuminations):
    """Illumination frequencies as a contiguous (count, 2) float32 array."""
    return np.ascontiguousarray(np.asarray(illuminations, dtype=np.float32).reshape(-1, 2))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def find_sideband(hologram, dc_exclusion: float = 0.0) -> Sideband:
    """Locate the +1 diffraction order in the spectrum of the (first) hologram: the strongest bin of
    the right half plane outside a disc of radius ``dc_exclusion`` around DC (N/8 when 0), refined to
    a fraction of a bin; positions in pixels relative to DC."""
    return _core.find_sideband(_Images(hologram, np.float32).stack, dc_exclusion)


def extract_fields(holograms, center=None, radius: float = 0.0, dc_exclusion: float = 0.0, output_size: int = 0,
                   backend: str = "cuda"):
    """Demodulate off-axis holograms into complex fields: the sideband at ``center`` (y, x pixels from
    DC; searched for with ``find_sideband`` when None) is cut out with a disc of ``radius`` (|center| / 3
    when 0), moved to the origin and transformed back on an ``output_size`` grid (the hologram's size
    when 0)."""
    h = _Images(holograms, np.float32)
    return h.give_back(_core.extract_fields(h.stack, center, radius, dc_exclusion, output_size, backend))


def field_ratio(sample, background):
    """Divide sample fields by background fields (a single background applies to every sample)."""
    s = _Images(sample, np.complex64)
    return s.give_back(_core.field_ratio(s.stack, _Images(background, np.complex64).stack))


def unwrap(phase, backend: str = "cuda"):
    """Unwrap phase images in the least-squares sense (the Neumann Poisson problem solved by cosine
    transforms), then add the constant that makes the result agree with the input modulo 2 pi."""
    p = _Images(phase, np.float32)
    return p.give_back(_core.unwrap(p.stack, backend))


def rytov(ratio, backend: str = "cuda"):
    """Complex Rytov phase of field ratios: log-amplitude plus i times the unwrapped phase, shifted by
    a multiple of 2 pi so that its mean over the image border lies in (-pi, pi]."""
    r = _Images(ratio, np.complex64)
    return r.give_back(_core.rytov(r.stack, backend))


def reconstruct(fields, illuminations, geometry: Geometry, nz: int = 0, iterations: int = 0, solver: str = "gp",
                gp_transform: str = "r2c", tv_weight: float = 1e-2, tv_inner: int = 10, mapping: str = "gather",
                backend: str = "cuda", return_filled: bool = False):
    """Refractive-index volume (nz, n, n) from Rytov fields (count, n, n), one per illumination.

    The fields' spectra are placed on their Ewald caps; ``iterations`` = 0 inverts that directly.
    Otherwise ``solver="gp"`` alternates the measured k-space data with a non-negative potential
    (Gerchberg-Papoulis; ``gp_transform`` "r2c" on half spectra or "c2c" on full ones) and
    ``solver="tv"`` runs FISTA with an isotropic total-variation penalty of weight ``tv_weight``,
    ``tv_inner`` dual steps per proximal step. ``nz`` (the field side when 0) must be even.
    ``return_filled`` adds the fraction of k-space voxels that data reached.
    """
    ri, filled = _core.reconstruct(_Images(fields, np.complex64).stack, _views(illuminations), geometry, nz,
                                   iterations, solver, gp_transform, tv_weight, tv_inner, mapping, backend)
    return (ri, filled) if return_filled else ri


class Pipeline:
    """The whole hologram-to-index chain for a fixed geometry, with everything it needs kept on the
    device between runs: plans, the background fields (from ``set_background``) and the k-space
    constants. A ``run`` moves the sample holograms in and the volume out once; ``upload_chunks``
    lets field extraction start on the first chunk while the rest are still in transfer.
    """

    def __init__(self, count: int, hologram_size: int, center, illuminations, geometry: Geometry,
                 radius: float = 0.0, output_size: int = 0, nz: int = 0, iterations: int = 0, solver: str = "gp",
                 gp_transform: str = "r2c", tv_weight: float = 1e-2, tv_inner: int = 10, mapping: str = "gather",
                 backend: str = "cuda", upload_chunks: int = 1):
        self._p = _core.Pipeline(count, hologram_size, tuple(center), radius, output_size, _views(illuminations),
                                 geometry, nz, iterations, solver, gp_transform, tv_weight, tv_inner, mapping, backend,
                                 upload_chunks)

    def set_background(self, backgrounds) -> None:
        """Take the background holograms (count, N, N); their fields are computed now and kept."""
        self._p.set_background(_f32(backgrounds))

    def run(self, holograms):
        """Reconstruct one stack of sample holograms (count, N, N); returns the volume (nz, n, n)."""
        return self._p.run(_f32(holograms))

    def run_stream(self, holograms):
        """Reconstruct many stacks (items, count, N, N) into (items, nz, n, n). Transfers of one stack
        hide behind the solve of the next, and every volume is bitwise what ``run`` returns for its
        stack; ``filled`` afterwards refers to the last one."""
        return self._p.run_stream(_f32(holograms))

    @property
    def filled(self) -> float:
        """Fraction of k-space voxels that the last run's data reached."""
        return self._p.filled

    @property
    def timings(self) -> dict[str, float]:
        """Stage times of the last run in milliseconds: device event intervals, ``total`` on the host."""
        return self._p.timings

    @property
    def setup_ms(self) -> float:
        """Time taken to build the pipeline, in milliseconds."""
        return self._p.setup_ms

    @property
    def device_bytes(self) -> int:
        """Device memory the pipeline holds."""
        return self._p.device_bytes


def circular_scan(count: int, na_illumination: float, geometry: Geometry):
    """Illumination frequencies (count, 2): the first view on axis, the others at equal steps around a
    cone of numerical aperture ``na_illumination``."""
    return _core.circular_scan(count, na_illumination, geometry)[0]


def render_phantom(spheres, geometry: Geometry, nz: int, n: int):
    """Sample the spheres' refractive index at the voxel centres of an (nz, n, n) grid of the
    geometry's pixel, the volume centred on the origin; later spheres paint over earlier ones."""
    return _core.render_phantom(list(spheres), geometry, nz, n)


def forward_fields(spheres, illuminations, geometry: Geometry, n: int, model: str = "rytov"):
    """Simulated field ratios u / u_in at the central plane (count, n, n), limited to the detection
    aperture: first Born (``"born"``), its Rytov form (``"rytov"``), or the exact scalar solution of a
    single sphere (``"exact"``)."""
    return _core.forward_fields(list(spheres), _views(illuminations), geometry, n, model)


def bpm_forward(ri, illuminations, geometry: Geometry, obliquity: bool = True, backend: str = "cuda"):
    """Field ratios (count, n, n) that the multi-slice beam-propagation model predicts for an index
    volume (nz, n, n)."""
    return _core.bpm_forward(_f32(ri), _views(illuminations), geometry, obliquity, backend)


def bpm_reconstruct(fields, illuminations, geometry: Geometry, initial, iterations: int = 20, batch: int = 0,
                    step: float = 1.0, tv_weight: float = 0.0, tv_inner: int = 10, obliquity: bool = True,
                    backend: str = "cuda", return_loss: bool = False):
    """Fit an index volume to measured field ratios through the beam-propagation model, starting from
    ``initial``: proximal gradient steps over all views (FISTA) or over batches of ``batch`` views,
    optionally with a total-variation term. ``return_loss`` adds the data misfit of every iteration."""
    ri, loss = _core.bpm_reconstruct(np.ascontiguousarray(fields, dtype=np.complex64), _views(illuminations),
                                     geometry, _f32(initial), iterations, batch, step, tv_weight, tv_inner, obliquity,
                                     backend)
    return (ri, np.asarray(loss)) if return_loss else ri


def synthesize_holograms(ratio, illuminations, geometry: Geometry, carrier=(5.0, 5.0),
                         reference_amplitude: float = 1.0, noise: float = 0.0, seed: int = 1):
    """Off-axis holograms of field ratios: the intensity of a tilted reference wave (amplitude
    ``reference_amplitude``, spatial frequency ``carrier``) plus the illuminated sample field, with
    additive Gaussian noise of standard deviation ``noise`` drawn from a generator seeded by ``seed``."""
    r = _Images(ratio, np.complex64)
    return r.give_back(_core.synthesize_holograms(r.stack, _views(illuminations), geometry, tuple(carrier),
                                                  reference_amplitude, noise, seed))
