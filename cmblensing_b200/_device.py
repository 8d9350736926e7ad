"""Move reference-shaped fields/operators to the GPU and back.

The inference functions run every step on the device (the engine's lensing
and FFT kernels plus float64 elementwise algebra on device tensors); host
numpy inputs are copied once at entry and results copied back at exit.
"""
from __future__ import annotations

import numpy as np
import torch


def _names(obj):
    return obj._matrix_names()


def device():
    if not torch.cuda.is_available():
        from ._native import NativeLibraryError
        raise NativeLibraryError("the LenseFlow engine needs a CUDA device; none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def to_device(obj, dev):
    upd = {}
    for n in _names(obj):
        m = getattr(obj, n)
        if not isinstance(m, torch.Tensor) or not m.is_cuda:
            m = torch.as_tensor(np.asarray(m) if not isinstance(m, torch.Tensor) else m, device=dev)
        if m.is_complex():
            m = m.to(torch.complex128)
        elif m.dtype != torch.float64:
            m = m.to(torch.float64)
        upd[n] = m
    return obj.replace(**upd)


def to_host(obj):
    return obj.replace(**{n: getattr(obj, n).cpu().numpy() for n in _names(obj)})


def on_device(fn):
    """Run ``fn`` with every field/operator argument on the GPU; return host results for host inputs."""
    import functools

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        host = False
        dev = None
        conv = []
        for a in args:
            if hasattr(a, "_matrix_names") and not isinstance(getattr(a, a._matrix_names()[0]), (int, float)):
                m = getattr(a, a._matrix_names()[0])
                if not (isinstance(m, torch.Tensor) and m.is_cuda):
                    host = True
                else:
                    dev = m.device
        dev = dev or device()
        for a in args:
            conv.append(to_device(a, dev) if hasattr(a, "_matrix_names") else a)
        out = fn(*conv, **kwargs)
        if not host:
            return out
        if isinstance(out, tuple):
            return tuple(_host_result(o) for o in out)
        return _host_result(out)
    return wrapper


def _host_result(out):
    if hasattr(out, "_matrix_names"):
        return to_host(out)
    if isinstance(out, torch.Tensor):
        return float(out) if out.dim() == 0 else out.cpu().numpy()
    return out
