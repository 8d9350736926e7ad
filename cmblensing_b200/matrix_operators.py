"""Fourier-diagonal operators with the reference's interface (cmb_lensing/matrix_operators.py:11-234).

``DiagonalScalar`` (T), ``DiagonalEB`` (EE, BB) and ``BlockTEB`` (TT, TE, ET,
EE, BB) keep the reference's attribute names, products, ``pinv`` and
``log_det``.  Matrices may be numpy arrays or torch tensors; the inference
functions move them to the device once per call.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .constants import NSIDE_DEFAULT, PIX_WIDTH_DEFAULT, THETA_PIX_DEFAULT
from .fields import FlatS0, FlatS02, FlatS2, fourier_weights_default

try:
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_torch(x):
    return torch is not None and isinstance(x, torch.Tensor)


def reciprocal_matrix(m):
    """util.py:45-47: 1/m with 0 -> 0."""
    if _is_torch(m):
        return torch.where(m != 0, 1.0 / torch.where(m != 0, m, torch.ones_like(m)), torch.zeros_like(m))
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(m != 0, 1.0 / np.where(m != 0, m, 1), 0.0)


def _logabs(m):
    if _is_torch(m):
        return torch.where(m != 0, torch.log(torch.abs(torch.where(m != 0, m, torch.ones_like(m)))),
                           torch.zeros_like(m, dtype=torch.float64))
    with np.errstate(divide="ignore"):
        return np.where(m != 0, np.log(np.abs(np.where(m != 0, m, 1))), 0.0)


def primal_log_det(m, w):
    """util.py:39-42."""
    if _is_torch(m):
        wt = torch.as_tensor(w, device=m.device)
        val = torch.sum(_logabs(m) * wt)
        sign = torch.prod(torch.sign(torch.where(m != 0, m, torch.ones_like(m))))
        return sign * val
    val = np.sum(_logabs(m) * w)
    sign = np.prod(np.sign(np.where(m != 0, m, 1)))
    return sign * val


@dataclasses.dataclass
class FieldOperator:
    nside: int = NSIDE_DEFAULT
    theta_pix: float = THETA_PIX_DEFAULT
    pix_width: float = PIX_WIDTH_DEFAULT
    fourier_weights: object = None

    def __post_init__(self):
        if self.fourier_weights is None:
            self.fourier_weights = fourier_weights_default(self.nside)

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    def __add__(self, other):
        if isinstance(other, self.__class__):
            return self.replace(**{n: getattr(self, n) + getattr(other, n) for n in self._matrix_names()})
        return self.replace(**{n: getattr(self, n) + other for n in self._matrix_names()})

    def __sub__(self, other):
        if isinstance(other, self.__class__):
            return self.replace(**{n: getattr(self, n) - getattr(other, n) for n in self._matrix_names()})
        return self.replace(**{n: getattr(self, n) - other for n in self._matrix_names()})


@dataclasses.dataclass
class DiagonalScalar(FieldOperator):
    """matrix_operators.py:46-63."""
    scalar_matrix: object = None

    def _matrix_names(self):
        return ["scalar_matrix"]

    def __mul__(self, other):
        if isinstance(other, (PixelMask, ComposedOperator)):
            return ComposedOperator([self]) * other
        if isinstance(other, DiagonalScalar):
            return self.replace(scalar_matrix=self.scalar_matrix * other.scalar_matrix)
        if isinstance(other, FlatS0):
            return other.replace(scalar_matrix=self.scalar_matrix * other.scalar_matrix)
        return self.replace(scalar_matrix=self.scalar_matrix * other)

    __rmul__ = __mul__


@dataclasses.dataclass
class DiagonalEB(FieldOperator):
    """matrix_operators.py:66-90."""
    matrix_EE: object = None
    matrix_BB: object = None

    def _matrix_names(self):
        return ["matrix_EE", "matrix_BB"]

    def __mul__(self, other):
        if isinstance(other, (PixelMask, ComposedOperator)):
            return ComposedOperator([self]) * other
        if isinstance(other, DiagonalEB):
            return self.replace(matrix_EE=self.matrix_EE * other.matrix_EE, matrix_BB=self.matrix_BB * other.matrix_BB)
        if isinstance(other, FlatS2):
            return other.replace(polar_matrix_1=self.matrix_EE * other.polar_matrix_1,
                                 polar_matrix_2=self.matrix_BB * other.polar_matrix_2)
        return self.replace(matrix_EE=self.matrix_EE * other, matrix_BB=self.matrix_BB * other)

    __rmul__ = __mul__


@dataclasses.dataclass
class BlockTEB(FieldOperator):
    """matrix_operators.py:93-148: [TT TE 0; ET EE 0; 0 0 BB]."""
    matrix_TT: object = None
    matrix_TE: object = None
    matrix_ET: object = None
    matrix_EE: object = None
    matrix_BB: object = None

    def _matrix_names(self):
        return ["matrix_TT", "matrix_TE", "matrix_ET", "matrix_EE", "matrix_BB"]

    def __mul__(self, other):
        s = self
        if isinstance(other, (PixelMask, ComposedOperator)):
            return ComposedOperator([self]) * other
        if isinstance(other, BlockTEB):
            o = other
            return s.replace(matrix_TT=s.matrix_TT * o.matrix_TT + s.matrix_TE * o.matrix_ET,
                             matrix_ET=s.matrix_ET * o.matrix_TT + s.matrix_EE * o.matrix_ET,
                             matrix_TE=s.matrix_TT * o.matrix_TE + s.matrix_TE * o.matrix_EE,
                             matrix_EE=s.matrix_ET * o.matrix_TE + s.matrix_EE * o.matrix_EE,
                             matrix_BB=s.matrix_BB * o.matrix_BB)
        if isinstance(other, FlatS02):
            return other.replace(scalar_matrix=s.matrix_TT * other.scalar_matrix + s.matrix_TE * other.polar_matrix_1,
                                 polar_matrix_1=s.matrix_ET * other.scalar_matrix + s.matrix_EE * other.polar_matrix_1,
                                 polar_matrix_2=s.matrix_BB * other.polar_matrix_2)
        return s.replace(**{n: getattr(s, n) * other for n in s._matrix_names()})

    def __rmul__(self, other):
        if isinstance(other, BlockTEB):
            return other.__mul__(self)
        return self.replace(**{n: getattr(self, n) * other for n in self._matrix_names()})


# ------------------------------------------------- map-space masks (extension)
@dataclasses.dataclass
class PixelMask(FieldOperator):
    """Multiplication by a real (N, N) map in pixel space, acting on Fourier fields.

    Not in the reference, whose masks are Fourier-diagonal (``DiagonalEB``);
    used for masks with holes.  On an EB (or T) Fourier field it applies
    qu2eb(fourier(m * map(eb2qu(f)))), so it slots into the reference's
    formulas (gradients.py:17-25) unchanged.  Products with diagonal operators
    become ``ComposedOperator``s applied right to left.
    """
    mask_map: object = None

    def _matrix_names(self):
        return ["mask_map"]

    def apply(self, field):
        from .fields import eb2qu, fourier, map, qu2eb
        mp = map(eb2qu(field))
        mp = mp.replace(**{n: getattr(mp, n) * self.mask_map for n in mp._matrix_names()})
        return qu2eb(fourier(mp))

    def __mul__(self, other):
        if isinstance(other, (FlatS0, FlatS2, FlatS02)):
            return self.apply(other)
        if isinstance(other, FieldOperator) or isinstance(other, ComposedOperator):
            return ComposedOperator([self]) * other
        return self.replace(mask_map=self.mask_map * other)

    def diagonal_like(self, op):
        """A Fourier-diagonal stand-in of the same kind as ``op`` with value sqrt(mean(m^2)) (for preconditioners)."""
        m = self.mask_map
        v = float((m * m).mean()) ** 0.5
        ones = lambda a: (a * 0 + 1) * v
        return op.replace(**{n: ones(getattr(op, n)) for n in op._matrix_names()})


class ComposedOperator:
    """A product of operators, applied right to left to a field."""

    def __init__(self, ops):
        self.ops = list(ops)

    def __mul__(self, other):
        if isinstance(other, (FlatS0, FlatS2, FlatS02)):
            out = other
            for op in reversed(self.ops):
                out = op * out
            return out
        if isinstance(other, ComposedOperator):
            return ComposedOperator(self.ops + other.ops)
        if isinstance(other, (FieldOperator, PixelMask)):
            return ComposedOperator(self.ops + [other])
        return ComposedOperator(self.ops[:-1] + [self.ops[-1] * other])


def pinv(op):
    """matrix_operators.py:205-234."""
    if isinstance(op, DiagonalScalar):
        return op.replace(scalar_matrix=reciprocal_matrix(op.scalar_matrix))
    if isinstance(op, DiagonalEB):
        return op.replace(matrix_EE=reciprocal_matrix(op.matrix_EE), matrix_BB=reciprocal_matrix(op.matrix_BB))
    if isinstance(op, BlockTEB):
        a, b, c, d = op.matrix_TT, op.matrix_TE, op.matrix_ET, op.matrix_EE
        rd = reciprocal_matrix(d)
        sc = reciprocal_matrix(a - b * rd * c)
        return op.replace(matrix_TT=sc, matrix_TE=-sc * b * rd, matrix_ET=-rd * c * sc,
                          matrix_EE=rd + rd * c * sc * b * rd, matrix_BB=reciprocal_matrix(op.matrix_BB))
    raise TypeError(type(op))


def log_det(op):
    """matrix_operators.py:175-200."""
    w = op.fourier_weights
    if isinstance(op, DiagonalScalar):
        return primal_log_det(op.scalar_matrix, w)
    if isinstance(op, DiagonalEB):
        return primal_log_det(op.matrix_EE, w) + primal_log_det(op.matrix_BB, w)
    if isinstance(op, BlockTEB):
        a, b, c, d = op.matrix_TT, op.matrix_TE, op.matrix_ET, op.matrix_EE
        return (primal_log_det(a, w) + primal_log_det(d - c * reciprocal_matrix(a) * b, w)
                + primal_log_det(op.matrix_BB, w))
    raise TypeError(type(op))
