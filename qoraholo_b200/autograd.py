"""The multi-slice BPM forward model as a differentiable torch operation.

``BpmModel(nz, n, illuminations, geometry)`` maps a refractive-index volume (nz, n, n) float32 on
the GPU to the field ratios (count, n, n) complex64 at z = 0 that the reference's ``bpm_forward``
computes (src/cuda/bpm.cu:157-174, src/bpm.cpp:10-60). Its backward pass is the hand-written
adjoint slice sweep of libqhk.so (qhk_bpm_plan_vjp): for an upstream gradient g it returns
Re(J^H g), which for g = y - data is the gradient of 1/2 |y - data|^2 -- the reference's bpm_vjp
(src/cuda/bpm.cu:250-272). Torch's convention for a real loss of complex outputs hands backward
exactly that g, so autograd losses built on the fields get the true gradient.

Memory: the forward keeps, per illumination, only the spectrum entering every
``checkpoint_every``-th slice; backward recomputes each segment of slices from its checkpoint before
sweeping it backwards (one extra forward pass), instead of storing the envelope at every slice
(8 n^2 nz bytes per illumination). ``checkpoint_every=0`` stores every envelope.

torch provides the device memory and the stream here; all arithmetic is in libqhk.so.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi

_VP = C.c_void_p
_I = C.c_int

_PROTOS = {
    "qhk_bpm_plan_create": (_I, [C.POINTER(_VP), _I, _I, _VP, _I, C.POINTER(capi.Geometry), _I, _I, _I]),
    "qhk_bpm_plan_forward": (_I, [_VP, _VP, _VP, _VP]),
    "qhk_bpm_plan_vjp": (_I, [_VP, _VP, _VP, _VP, _VP]),
    "qhk_bpm_plan_device_bytes": (C.c_size_t, [_VP]),
    "qhk_bpm_plan_destroy": (_I, [_VP]),
}


def _lib():
    lib = capi.lib()
    for name, (res, args) in _PROTOS.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


class BpmPlan:
    """qhk_bpm_plan_*: the BPM forward model and its vector-Jacobian product on device pointers."""

    def __init__(self, nz, n, illuminations, geometry, obliquity=True, chunk=0, checkpoint_every=16):
        self._il = np.ascontiguousarray(np.reshape(illuminations, (-1, 2)), np.float32)
        self.nz, self.n, self.count = int(nz), int(n), int(self._il.shape[0])
        self._h = _VP()
        capi.check(_lib().qhk_bpm_plan_create(C.byref(self._h), self.nz, self.n, capi.host_ptr(self._il), self.count,
                                              C.byref(capi.geometry(geometry)), int(bool(obliquity)), int(chunk),
                                              int(checkpoint_every)))

    def forward(self, d_ri, d_fields, stream=0):
        capi.check(_lib().qhk_bpm_plan_forward(self._h, _VP(d_ri), _VP(d_fields), _VP(stream)))

    def vjp(self, d_ri, d_grad_fields, d_grad_ri, stream=0):
        capi.check(_lib().qhk_bpm_plan_vjp(self._h, _VP(d_ri), _VP(d_grad_fields), _VP(d_grad_ri), _VP(stream)))

    @property
    def device_bytes(self):
        return int(_lib().qhk_bpm_plan_device_bytes(self._h))

    def close(self):
        if self._h:
            capi.check(_lib().qhk_bpm_plan_destroy(self._h))
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _checked(ri, model):
    if not (ri.is_cuda and ri.dtype == torch.float32):
        raise TypeError("BpmModel: the volume must be a float32 CUDA tensor")
    if tuple(ri.shape) != (model.nz, model.n, model.n):
        raise ValueError(f"BpmModel: the volume must have shape {(model.nz, model.n, model.n)}")
    return ri.contiguous()


class _BpmFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ri, model):
        ri = _checked(ri, model)
        fields = torch.empty((model.count, model.n, model.n), dtype=torch.complex64, device=ri.device)
        model.plan.forward(ri.data_ptr(), fields.data_ptr(), torch.cuda.current_stream(ri.device).cuda_stream)
        model._generation += 1
        ctx.generation = model._generation
        ctx.model = model
        ctx.save_for_backward(ri)
        return fields

    @staticmethod
    def backward(ctx, grad_fields):
        (ri,) = ctx.saved_tensors
        model = ctx.model
        stream = torch.cuda.current_stream(ri.device).cuda_stream
        if model._generation != ctx.generation:
            # Another forward replaced the checkpoints: rebuild them for this volume.
            scratch = torch.empty((model.count, model.n, model.n), dtype=torch.complex64, device=ri.device)
            model.plan.forward(ri.data_ptr(), scratch.data_ptr(), stream)
            model._generation += 1
            ctx.generation = model._generation
        g = grad_fields.to(torch.complex64).contiguous()
        grad = torch.empty_like(ri)
        model.plan.vjp(ri.data_ptr(), g.data_ptr(), grad.data_ptr(), stream)
        return grad, None


class BpmModel(torch.nn.Module):
    """Differentiable BPM: ``model(ri)`` -> field ratios (count, n, n) complex64 at z = 0.

    Same model and geometry conventions as ``qoraholo_b200.bpm_forward`` (dz = pixel, the volume
    centred on z = 0 of the detection plane, ``obliquity`` weighting). ``checkpoint_every`` slices per
    stored spectrum; ``chunk`` illuminations per device pass (0: all)."""

    def __init__(self, nz, n, illuminations, geometry, obliquity=True, checkpoint_every=16, chunk=0):
        super().__init__()
        if checkpoint_every == 0 and chunk not in (0, len(np.reshape(illuminations, (-1, 2)))):
            raise ValueError("BpmModel: storing every envelope needs all illuminations in one chunk")
        self.plan = BpmPlan(nz, n, illuminations, geometry, obliquity, chunk, checkpoint_every)
        self.nz, self.n, self.count = self.plan.nz, self.plan.n, self.plan.count
        self._generation = 0

    def forward(self, ri):
        return _BpmFunction.apply(ri, self)
