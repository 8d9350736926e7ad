"""Drop-in ``lense_flow`` (cmb_lensing/lense_flow.py:289-292) backed by the CUDA engine.

Same signature and defaults as the reference: ``lense_flow(field, phi, n=10,
direction=1, adjoint=False)`` lenses every matrix of a MAP-basis T / QU /
TQU field with ``field.pix_width`` and returns ``field.replace(...)``.  phi
may be a MAP ``(N, N)`` or a FOURIER ``(N, N/2+1)`` matrix, as in the
reference (lense_flow.py:299-302).  Host numpy inputs are copied to the GPU
and the result is returned as float64 numpy; torch CUDA inputs stay on the
device.  All components of the field are integrated in one batched launch
sequence that reads the phi derivatives once per row tile.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine
from .constants import FORWARD_LENSE, INVERSE_LENSE  # noqa: F401


def _device():
    if not torch.cuda.is_available():
        from ._native import NativeLibraryError
        raise NativeLibraryError("the LenseFlow engine needs a CUDA device; none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def lense_flow(field, phi, n=10, direction=1, adjoint=False, precision="f32"):
    names = field._matrix_names()
    mats = [getattr(field, nm) for nm in names]
    host = not isinstance(mats[0], torch.Tensor)
    dev = mats[0].device if not host and mats[0].is_cuda else _device()
    f = torch.stack([torch.as_tensor(m, device=dev) for m in mats]).unsqueeze(0)
    if f.dtype not in (torch.float32, torch.float64):
        f = f.to(torch.float64)
    pm = phi.scalar_matrix
    pt = torch.as_tensor(pm, device=dev)
    pt = pt.to(torch.complex128) if pt.is_complex() else pt.to(torch.float64)
    out = engine.lense_flow_batch(f, pt.unsqueeze(0), field.pix_width, n=n, direction=direction, adjoint=adjoint,
                                  precision=precision)
    if host:
        arr = out[0].to(torch.float64).cpu().numpy()
        upd = {nm: arr[i] for i, nm in enumerate(names)}
    else:
        upd = {nm: out[0, i] for i, nm in enumerate(names)}
    return field.replace(**upd)
