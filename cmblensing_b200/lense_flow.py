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
        engine.check_timeouts("lense_flow")
        upd = {nm: arr[i] for i, nm in enumerate(names)}
    else:
        upd = {nm: out[0, i] for i, nm in enumerate(names)}
    return field.replace(**upd)


def _stack(field, dev):
    mats = [torch.as_tensor(getattr(field, nm), device=dev) for nm in field._matrix_names()]
    t = torch.stack(mats).unsqueeze(0)
    return t if t.dtype in (torch.float32, torch.float64) else t.real.to(torch.float64)


def lense_flow_backwards(transformed_field, phi, cotangent, n=10, direction=1, swap_qu=True, precision="f32",
                         scheme="reference", field=None):
    """The reference's custom-VJP backward pass (cmb_lensing/lense_flow.py:23-46).

    Integrates (f, delta_f, delta_phi) from the lensed field in the opposite
    time direction on the GPU (lf_lense_flow_vjp) and returns
    ``(undo_inner_product(delta_field), undo_inner_product(delta_phi))``.
    With ``swap_qu`` the Q/U matrices of delta_field are returned swapped, as
    the reference's output_like_input writes them (lense_flow.py:143-144,
    151-152); pass ``swap_qu=False`` for the mathematically ordered result.
    ``scheme="exact"`` runs the checkpointed reverse pass instead
    (lf_lense_flow_vjp_ckpt): it needs ``field``, the unlensed MAP-basis field
    that ``transformed_field`` came from (the reference's VJP residuals hold it
    too, lense_flow.py:10-21), and returns the exact gradient of the discrete
    lens for delta_phi.
    """
    from .fields import FlatS0, undo_inner_product
    names = transformed_field._matrix_names()
    m0 = getattr(transformed_field, names[0])
    host = not isinstance(m0, torch.Tensor)
    dev = m0.device if not host and m0.is_cuda else _device()
    fl = _stack(transformed_field, dev).to(torch.float64)
    ct = _stack(cotangent, dev).to(torch.float64)
    pm = torch.as_tensor(phi.scalar_matrix, device=dev)
    fourier_phi = pm.shape[-1] != pm.shape[-2]
    pm = pm.to(torch.complex128) if fourier_phi else pm.to(torch.float64)
    plan = engine.get_plan(fl.shape[-1], fl.shape[1], phi.pix_width, precision, device=dev)
    planes = plan.phi_planes(pm.unsqueeze(0), check_det=False)
    basis = "fourier" if fourier_phi else "map"
    if scheme == "exact":
        if field is None:
            raise ValueError("scheme='exact' needs the unlensed field (field=...)")
        df, dphi = plan.lense_flow_vjp_ckpt(_stack(field, dev).to(torch.float64), ct, planes, n=n,
                                            direction=direction, phi_basis=basis)
    elif scheme == "reference":
        df, dphi = plan.lense_flow_vjp(fl, ct, planes, n=n, direction=direction, phi_basis=basis)
    else:
        raise ValueError(f"unknown reverse-pass scheme {scheme!r}")
    comps = [df[0, i] for i in range(len(names))]
    if swap_qu and not isinstance(transformed_field, FlatS0):
        comps[-2], comps[-1] = comps[-1], comps[-2]
    if host:
        torch.cuda.current_stream(dev).synchronize()
        engine.check_timeouts("lense_flow_backwards")
    conv = (lambda t: t.cpu().numpy()) if host else (lambda t: t)
    dfield = transformed_field.replace(**{nm: conv(c) for nm, c in zip(names, comps)})
    dphi_field = phi.replace(scalar_matrix=conv(dphi[0]))
    return undo_inner_product(dfield), undo_inner_product(dphi_field)
