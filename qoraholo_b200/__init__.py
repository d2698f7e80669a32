"""Holotomography (optical diffraction tomography) reconstruction on NVIDIA B200.

Drop-in for the ``qoraholo`` Python package: the same functions, arguments and return values
(python/qoraholo/__init__.py of QoraHolo), computed by hand-written sm_100a CUDA kernels behind
the C ABI of ``libqhk.so`` (include/qoraholo_b200.h). ``backend`` defaults to ``"cuda"``, the only
backend of this build; ``"cpu"`` raises.

Arrays are numpy, centre-origin, square with even sides. Functions that work on images accept a
single 2D image or a 3D stack (count, n, n) and return the same rank. Lengths are micrometres,
spatial frequencies cycles per micrometre.
"""

from __future__ import annotations

import numpy as np

try:
    from . import _core  # noqa: E402
except ImportError as e:  # fail loudly: there is no fallback implementation
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


def _stack(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.ndim == 2:
        return a[None], True
    if a.ndim != 3:
        raise ValueError(f"expected a 2D image or a 3D stack, got {a.ndim} dimensions")
    return a, False


def _unstack(a, single):
    return a[0] if single else a


def _illum(illuminations):
    return np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), dtype=np.float32)


def find_sideband(hologram, dc_exclusion: float = 0.0) -> Sideband:
    """Peak of the +1 sideband (x > 0 half plane) of the first hologram, in pixels from DC."""
    h, _ = _stack(hologram, np.float32)
    return _core.find_sideband(h, dc_exclusion)


def extract_fields(holograms, center=None, radius: float = 0.0, dc_exclusion: float = 0.0, output_size: int = 0,
                   backend: str = "cuda"):
    """Off-axis hologram(s) to complex field(s).

    ``center`` is the sideband centre (y, x) in pixels from DC; detected when omitted. ``radius``
    defaults to |center| / 3, ``output_size`` to the hologram side.
    """
    h, single = _stack(holograms, np.float32)
    return _unstack(_core.extract_fields(h, center, radius, dc_exclusion, output_size, backend), single)


def field_ratio(sample, background):
    """sample / background; background is one field or one per sample field."""
    s, single = _stack(sample, np.complex64)
    b, _ = _stack(background, np.complex64)
    return _unstack(_core.field_ratio(s, b), single)


def unwrap(phase, backend: str = "cuda"):
    """Least-squares unwrapping (Ghiglia & Romero 1994), congruent to the input mod 2 pi."""
    p, single = _stack(phase, np.float32)
    return _unstack(_core.unwrap(p, backend), single)


def rytov(ratio, backend: str = "cuda"):
    """log|r| + i unwrap(arg r), with the mean phase on the image border in (-pi, pi]."""
    r, single = _stack(ratio, np.complex64)
    return _unstack(_core.rytov(r, backend), single)


def reconstruct(fields, illuminations, geometry: Geometry, nz: int = 0, iterations: int = 0, solver: str = "gp",
                gp_transform: str = "r2c", tv_weight: float = 1e-2, tv_inner: int = 10, mapping: str = "gather",
                backend: str = "cuda", return_filled: bool = False):
    """Rytov fields (count, n, n) to a refractive-index volume (nz, n, n).

    ``solver="gp"``: Gerchberg-Papoulis with n >= n_medium (``gp_transform`` "r2c" half spectra or
    "c2c"); ``solver="tv"``: FISTA with a TV term of weight ``tv_weight`` on n^2 - n_medium^2 and
    ``tv_inner`` FGP steps per iteration. ``return_filled`` also returns the fraction of k-space
    voxels that received data.
    """
    f, _ = _stack(fields, np.complex64)
    ri, filled = _core.reconstruct(f, _illum(illuminations), geometry, nz, iterations, solver, gp_transform,
                                   tv_weight, tv_inner, mapping, backend)
    return (ri, filled) if return_filled else ri


class Pipeline:
    """Holograms to refractive index with device state allocated once.

    The background fields stay on the device; each ``run`` does one upload of the sample holograms
    and one download of the volume, from page-locked buffers. ``upload_chunks`` splits the upload
    so field extraction overlaps it.
    """

    def __init__(self, count: int, hologram_size: int, center, illuminations, geometry: Geometry,
                 radius: float = 0.0, output_size: int = 0, nz: int = 0, iterations: int = 0, solver: str = "gp",
                 gp_transform: str = "r2c", tv_weight: float = 1e-2, tv_inner: int = 10, mapping: str = "gather",
                 backend: str = "cuda", upload_chunks: int = 1):
        self._p = _core.Pipeline(count, hologram_size, tuple(center), radius, output_size, _illum(illuminations),
                                 geometry, nz, iterations, solver, gp_transform, tv_weight, tv_inner, mapping, backend,
                                 upload_chunks)

    def set_background(self, backgrounds) -> None:
        """Background holograms (count, N, N); their fields are extracted once and kept."""
        self._p.set_background(np.ascontiguousarray(backgrounds, dtype=np.float32))

    def run(self, holograms):
        """Sample holograms (count, N, N) to the index volume (nz, n, n)."""
        return self._p.run(np.ascontiguousarray(holograms, dtype=np.float32))

    def run_stream(self, holograms):
        """A stream of stacks (items, count, N, N) to volumes (items, nz, n, n): each stack's upload
        and each volume's download overlap the solve of its neighbour; each volume is bitwise what
        ``run`` gives for its stack. ``filled`` is then the last stack's."""
        return self._p.run_stream(np.ascontiguousarray(holograms, dtype=np.float32))

    @property
    def filled(self) -> float:
        return self._p.filled

    @property
    def timings(self) -> dict[str, float]:
        """Milliseconds per stage of the last run (device event intervals; ``total`` is host time)."""
        return self._p.timings

    @property
    def setup_ms(self) -> float:
        return self._p.setup_ms

    @property
    def device_bytes(self) -> int:
        return self._p.device_bytes


def circular_scan(count: int, na_illumination: float, geometry: Geometry):
    """Normal incidence, then count - 1 directions evenly spaced on a circle: (count, 2)."""
    return _core.circular_scan(count, na_illumination, geometry)[0]


def render_phantom(spheres, geometry: Geometry, nz: int, n: int):
    """Refractive index of the spheres at voxel centres, (nz, n, n)."""
    return _core.render_phantom(list(spheres), geometry, nz, n)


def forward_fields(spheres, illuminations, geometry: Geometry, n: int, model: str = "rytov"):
    """Field ratios u / u_in at z = 0, (count, n, n), band-limited to the detection NA."""
    return _core.forward_fields(list(spheres), _illum(illuminations), geometry, n, model)


def bpm_forward(ri, illuminations, geometry: Geometry, obliquity: bool = True, backend: str = "cuda"):
    """Refractive index (nz, n, n) to field ratios (count, n, n) by multi-slice beam propagation."""
    return _core.bpm_forward(np.ascontiguousarray(ri, dtype=np.float32), _illum(illuminations), geometry, obliquity,
                             backend)


def bpm_reconstruct(fields, illuminations, geometry: Geometry, initial, iterations: int = 20, batch: int = 0,
                    step: float = 1.0, tv_weight: float = 0.0, tv_inner: int = 10, obliquity: bool = True,
                    backend: str = "cuda", return_loss: bool = False):
    """Field ratios (count, n, n) to refractive index by gradient descent on the BPM."""
    ri, loss = _core.bpm_reconstruct(np.ascontiguousarray(fields, dtype=np.complex64), _illum(illuminations), geometry,
                                     np.ascontiguousarray(initial, dtype=np.float32), iterations, batch, step,
                                     tv_weight, tv_inner, obliquity, backend)
    return (ri, np.asarray(loss)) if return_loss else ri


def synthesize_holograms(ratio, illuminations, geometry: Geometry, carrier=(5.0, 5.0),
                         reference_amplitude: float = 1.0, noise: float = 0.0, seed: int = 1):
    """|R + u_in * ratio|^2 + Gaussian noise, with R = a exp(-2 pi i carrier . r)."""
    r, single = _stack(ratio, np.complex64)
    out = _core.synthesize_holograms(r, _illum(illuminations), geometry, tuple(carrier), reference_amplitude, noise,
                                     seed)
    return _unstack(out, single)
