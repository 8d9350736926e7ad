"""Flat-sky field containers with the reference's interface (cmb_lensing/fields.py:15-227).

``FlatS0`` (T), ``FlatS2`` (Q,U or E,B) and ``FlatS02`` (T,Q,U or T,E,B) carry
the same attribute names, defaults and ``replace`` semantics as the
reference's flax pytrees, so code written against the reference reads the
same.  Matrices may be numpy arrays (host) or torch tensors (host or CUDA).

``map``/``fourier``/``eb2qu``/``qu2eb`` are the reference's basis and
parametrization conversions (fields.py:159-226, util.py:140-172); they are
format conversions around the lensing operator, not part of it.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .constants import (ARCMIN_PER_DEGREE, NSIDE_DEFAULT, PIX_WIDTH_DEFAULT, THETA_PIX_DEFAULT, Basis,
                        Parametrization)

try:  # torch is optional for host-only use of the containers
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_torch(x):
    return torch is not None and isinstance(x, torch.Tensor)


def fourier_weights_default(nside=NSIDE_DEFAULT):
    """2 with 0.5 at the DC/Nyquist columns (constants.py:21)."""
    w = 2.0 * np.ones(nside // 2 + 1, dtype=np.complex128)
    w[0] = 0.5
    w[-1] = 0.5
    return w


def get_fourier_weights(field_shape):
    """2 with 1 at the DC/Nyquist columns (util.py:90-96)."""
    rows = field_shape[0]
    w = 2.0 * np.ones(rows // 2 + 1, dtype=np.complex128)
    w[0] = 1.0
    w[-1] = 1.0
    return w


@dataclasses.dataclass
class Field:
    nside: int = NSIDE_DEFAULT
    theta_pix: float = THETA_PIX_DEFAULT
    pix_width: float = PIX_WIDTH_DEFAULT
    basis: int = Basis.FOURIER
    fourier_weights: object = None

    def __post_init__(self):
        if self.fourier_weights is None:
            self.fourier_weights = fourier_weights_default(self.nside)

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    def _matrix_names(self):
        raise NotImplementedError

    def _binop(self, other, op):
        if isinstance(other, self.__class__):
            upd = {n: op(getattr(self, n), getattr(other, n)) for n in self._matrix_names()}
        else:
            upd = {n: op(getattr(self, n), other) for n in self._matrix_names()}
        return self.replace(**upd)

    def __add__(self, o):
        return self._binop(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._binop(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._binop(o, lambda a, b: b - a)

    def __mul__(self, o):
        return self._binop(o, lambda a, b: a * b)

    __rmul__ = __mul__

    def __truediv__(self, o):
        return self._binop(o, lambda a, b: a / b)

    def __rtruediv__(self, o):
        return self._binop(o, lambda a, b: b / a)


@dataclasses.dataclass
class FlatS0(Field):
    scalar_matrix: object = None
    parametrization: int = Parametrization.T

    def _matrix_names(self):
        return ["scalar_matrix"]


@dataclasses.dataclass
class FlatS2(Field):
    polar_matrix_1: object = None
    polar_matrix_2: object = None
    parametrization: int = Parametrization.EB

    def _matrix_names(self):
        return ["polar_matrix_1", "polar_matrix_2"]


@dataclasses.dataclass
class FlatS02(Field):
    scalar_matrix: object = None
    polar_matrix_1: object = None
    polar_matrix_2: object = None
    parametrization: int = Parametrization.EB

    def _matrix_names(self):
        return ["scalar_matrix", "polar_matrix_1", "polar_matrix_2"]


# ------------------------------------------------------------- conversions
def _fft_plan(m):
    from . import engine
    return engine.get_plan(m.shape[-2], 1, 1.0, "f64", device=m.device)


def _rfft2(m):
    """rfft2; CUDA tensors go through the engine's float64 FFT kernels (lf_rfft2)."""
    if _is_torch(m):
        if m.is_cuda:
            x = m if m.dtype in (torch.float32, torch.float64) else m.real
            return _fft_plan(m).rfft2(x.reshape((-1,) + tuple(m.shape[-2:]))).reshape(
                tuple(m.shape[:-1]) + (m.shape[-1] // 2 + 1,))
        return torch.fft.rfft2(m)
    return np.fft.rfft2(m)


def _irfft2(m):
    """irfft2; CUDA tensors go through the engine's float64 FFT kernels (lf_irfft2)."""
    n = m.shape[-2]
    if _is_torch(m):
        if m.is_cuda:
            return _fft_plan(m).irfft2(m.reshape((-1,) + tuple(m.shape[-2:]))).reshape(tuple(m.shape[:-1]) + (n,))
        return torch.fft.irfft2(m, s=(n, n))
    return np.fft.irfft2(m, s=(n, n))


def fourier(field):
    """fields.py:159-163."""
    return field.replace(basis=Basis.FOURIER, **{n: _rfft2(getattr(field, n)) for n in field._matrix_names()})


def map(field):  # noqa: A001  (name kept from fields.py:168)
    """fields.py:168-172."""
    return field.replace(basis=Basis.MAP, **{n: _irfft2(getattr(field, n)) for n in field._matrix_names()})


_ANGLES = {}


def _eb_angle(nside, theta_pix, like=None):
    """arctan2(lx, ly) on the rfft2 grid with the reference's Nyquist flip (util.py:140-149)."""
    key = (int(nside), float(theta_pix))
    a = _ANGLES.get(key)
    if a is None:
        d = math.radians(theta_pix / ARCMIN_PER_DEGREE)
        lx = 2 * np.pi * np.fft.rfftfreq(nside, d)
        ly = 2 * np.pi * np.fft.fftfreq(nside, d)
        lx, ly = np.meshgrid(lx, ly)
        lx[: nside // 2 + 1, -1] *= -1  # util.py:143
        a = np.arctan2(lx, ly)
        _ANGLES[key] = a
    if _is_torch(like):
        dkey = key + (str(like.device),)
        t = _ANGLES.get(dkey)
        if t is None:
            t = (torch.as_tensor(np.cos(2 * a), device=like.device), torch.as_tensor(np.sin(2 * a), device=like.device))
            _ANGLES[dkey] = t
        return t
    return np.cos(2 * a), np.sin(2 * a)


def eb2qu(field):
    """fields.py:178-199 with util.py:140-149."""
    if isinstance(field, FlatS0):
        return field
    e, b = field.polar_matrix_1, field.polar_matrix_2
    c2a, s2a = _eb_angle(field.nside, field.theta_pix, e)
    return field.replace(polar_matrix_1=-e * c2a + b * s2a, polar_matrix_2=-e * s2a - b * c2a,
                         parametrization=Parametrization.QU)


def qu2eb(field):
    """fields.py:203-226 with util.py:152-161."""
    if isinstance(field, FlatS0):
        return field
    q, u = field.polar_matrix_1, field.polar_matrix_2
    c2a, s2a = _eb_angle(field.nside, field.theta_pix, q)
    return field.replace(polar_matrix_1=-q * c2a - u * s2a, polar_matrix_2=q * s2a - u * c2a,
                         parametrization=Parametrization.EB)


def undo_inner_product(field):
    """fields.py:147-154: identity for Fourier-shaped matrices, else irfft2(conj(rfft2(m) / w) N^2)."""
    def _undo(m):
        if m.shape[-2] != m.shape[-1]:
            return m
        w = field.fourier_weights
        if _is_torch(m):
            w = torch.as_tensor(w, device=m.device)
            return _irfft2(torch.conj(_rfft2(m) / w) * field.nside ** 2)
        return _irfft2(np.conj(_rfft2(m) / w) * field.nside ** 2)
    return field.replace(**{n: _undo(getattr(field, n)) for n in field._matrix_names()})


def dot(field_1, field_2):
    """fields.py:137-142: Re sum conj(a) b w / N^2 with the first field's weights."""
    s = 0.0
    w = field_1.fourier_weights
    for n in field_1._matrix_names():
        a, b = getattr(field_1, n), getattr(field_2, n)
        if _is_torch(a):
            wt = torch.as_tensor(w, device=a.device)
            s = s + torch.real(torch.sum(torch.conj(a) * b * wt)) / field_1.nside ** 2
        else:
            s = s + float(np.real(np.sum(np.conj(a) * b * w))) / field_1.nside ** 2
    return s
