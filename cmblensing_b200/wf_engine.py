"""Device-resident Wiener filter: the reference's PCG (wiener_filter.py:52-104) with precomputed operators.

Every chain of EB<->QU rotations (util.py:140-161) and Fourier-diagonal
operators (matrix_operators.py) is, per Fourier mode, a real C x C matrix.
``DeviceWienerFilter`` builds those matrices once per problem, so one
application of A f = gradf_logpdf(f, d = 0) is

    q  = irfft2(R^T x)                          R: qu2eb rotation per mode
    y  = rfft2(L q)                              L: LenseFlow on the engine
    h  = W y                                     W = R^T B M Cn^-1 M B R (or the
                                                 map-space mask chain)
    z  = rfft2(L^T irfft2(h))                    L^T: adjoint LenseFlow
    Ax = -(R z + Cf^-1 x)

with the FFTs and lensing on the engine's kernels, the phi derivatives
computed once, the CG scalars kept on the device (no host round trip per
iteration) and one host synchronisation per convergence check.  Optional
true-residual replacement every ``refine_every`` iterations uses the FP64
engine for b - A x.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import engine
from ._device import device, to_device
from .fields import FlatS0, FlatS02, FlatS2, _eb_angle, map as to_map
from .matrix_operators import BlockTEB, DiagonalEB, DiagonalScalar, PixelMask, pinv


def _ncomp(field):
    return 1 if isinstance(field, FlatS0) else (2 if isinstance(field, FlatS2) else 3)


def _op_matrix(op, C, like):
    """(C, C, N, N/2+1) float64 per-mode matrix of a Fourier-diagonal operator."""
    N, H = like.shape[-2], like.shape[-1]
    W = torch.zeros((C, C, N, H), dtype=torch.float64, device=like.device)
    r = lambda m: torch.as_tensor(m, device=like.device).real.to(torch.float64) if torch.is_tensor(m) \
        else torch.as_tensor(np.real(np.asarray(m)), device=like.device)
    if isinstance(op, DiagonalScalar):
        W[0, 0] = r(op.scalar_matrix)
        if C > 1:
            raise TypeError("DiagonalScalar operator on a polarised field")
    elif isinstance(op, DiagonalEB):
        o = C - 2
        W[o, o] = r(op.matrix_EE)
        W[o + 1, o + 1] = r(op.matrix_BB)
    elif isinstance(op, BlockTEB):
        W[0, 0], W[0, 1] = r(op.matrix_TT), r(op.matrix_TE)
        W[1, 0], W[1, 1] = r(op.matrix_ET), r(op.matrix_EE)
        W[2, 2] = r(op.matrix_BB)
    else:
        raise TypeError(type(op))
    return W


def _mm(A, B):
    """Per-mode matrix product of (C, C, N, H) matrices."""
    return torch.einsum("ijnh,jknh->iknh", A, B)


class DeviceWienerFilter:
    """The Wiener filter of one problem, with operators, phi planes and buffers resident on the GPU."""

    def __init__(self, phi, data, field_covariance, noise_covariance, mask, beam, n=10, precision="f32"):
        dev = device()
        self.dev = dev
        args = [to_device(o, dev) for o in (phi, data, field_covariance, noise_covariance, beam)]
        phi, data, Cf, Cn, B = args
        self.data = data
        self.C = C = _ncomp(data)
        self.N = N = data.nside
        self.pw = data.pix_width
        self.n = n
        self.precision = precision
        first = getattr(data, data._matrix_names()[0])
        self.weights = torch.as_tensor(np.real(np.asarray(data.fourier_weights)), device=dev)
        # rotation qu2eb per mode (identity on T)
        R = torch.zeros((C, C, N, N // 2 + 1), dtype=torch.float64, device=dev)
        if C == 1:
            R[0, 0] = 1.0
        else:
            c2a, s2a = _eb_angle(N, data.theta_pix, first)
            o = C - 2
            if C == 3:
                R[0, 0] = 1.0
            R[o, o], R[o, o + 1] = -c2a, -s2a
            R[o + 1, o], R[o + 1, o + 1] = s2a, -c2a
        RT = R.transpose(0, 1).contiguous()
        self.R, self.RT = R, RT
        Cn_inv = _op_matrix(pinv(Cn), C, first)
        Bm = _op_matrix(B, C, first)
        self.Cf_inv = _op_matrix(pinv(Cf), C, first).to(torch.complex128)
        self.pixel_mask = None
        if isinstance(mask, PixelMask):
            self.pixel_mask = to_device(mask, dev).mask_map
            mdiag = _op_matrix(mask.diagonal_like(B), C, first)
            self.W_b = _mm(RT, _mm(Bm, R)).to(torch.complex128)          # QU -> QU through B
            self.W_n = _mm(RT, _mm(Cn_inv, R)).to(torch.complex128)      # QU -> QU through Cn^-1
            self._b_parts = (_mm(RT, Cn_inv).to(torch.complex128), _mm(Bm, R).to(torch.complex128))
            Mm = mdiag
        else:
            Mm = _op_matrix(mask, C, first)
            data_op = _mm(Bm, _mm(Mm, _mm(Cn_inv, _mm(Mm, Bm))))
            self.W_data = _mm(RT, _mm(data_op, R)).to(torch.complex128)   # QU -> QU
            self._bm_cn = _mm(Bm, _mm(Mm, Cn_inv)).to(torch.complex128)    # EB -> EB, for b
        P = _op_matrix(pinv(Cf), C, first) + _mm(Bm, _mm(Mm, _mm(Cn_inv, _mm(Mm, Bm))))
        self.P_inv = self._invert(P).to(torch.complex128)
        self.R_c, self.RT_c = R.to(torch.complex128), RT.to(torch.complex128)
        phimap = to_map(phi).scalar_matrix.to(torch.float64).unsqueeze(0)  # gradients.py:17 uses map(phi)
        self.phimap = phimap
        self.plan = engine.get_plan(N, C, self.pw, precision, device=dev)
        self.planes = engine.cached_phi_planes(self.plan, phimap)
        self.fft = engine.get_plan(N, 1, self.pw, "f64", device=dev)
        self._plan64 = None

    # ----------------------------------------------------------- pieces
    @staticmethod
    def _invert(P):
        """Per-mode pseudo-inverse of a block-diagonal C x C matrix (reciprocal with 0 -> 0, Schur for TE)."""
        C = P.shape[0]
        out = torch.zeros_like(P)
        rec = lambda a: torch.where(a != 0, 1.0 / torch.where(a != 0, a, torch.ones_like(a)), torch.zeros_like(a))
        if C == 1:
            out[0, 0] = rec(P[0, 0])
        elif C == 2:
            out[0, 0], out[1, 1] = rec(P[0, 0]), rec(P[1, 1])
        else:  # [TT TE 0; ET EE 0; 0 0 BB] as matrix_operators.py:222-234
            a, b, c, d = P[0, 0], P[0, 1], P[1, 0], P[1, 1]
            rd = rec(d)
            s = rec(a - b * rd * c)
            out[0, 0], out[0, 1], out[1, 0], out[1, 1] = s, -s * b * rd, -rd * c * s, rd + rd * c * s * b * rd
            out[2, 2] = rec(P[2, 2])
        return out

    @staticmethod
    def _apply(W, X):
        return torch.einsum("ijnh,jnh->inh", W, X)

    def _irfft2(self, X):
        return self.fft.irfft2(X)

    def _rfft2(self, X):
        return self.fft.rfft2(X)

    def _lens(self, q, adjoint, prec):
        if prec == self.precision:
            plan, planes = self.plan, self.planes
        else:
            if self._plan64 is None:
                self._plan64 = engine.get_plan(self.N, self.C, self.pw, prec, device=self.dev)
                self._planes64 = engine.cached_phi_planes(self._plan64, self.phimap)
            plan, planes = self._plan64, self._planes64
        return plan.lense_flow(q.unsqueeze(0), planes, n=self.n, adjoint=adjoint)[0]

    def _mask_chain(self, y):
        """QU spectra -> W y through the map-space mask: B, m, Cn^-1, m, B."""
        m = self.pixel_mask
        t = self._apply(self.W_b, y)
        t = self._rfft2(self._irfft2(t) * m)
        t = self._apply(self.W_n, t)
        t = self._rfft2(self._irfft2(t) * m)
        return self._apply(self.W_b, t)

    def apply_A(self, x, prec=None):
        """A x = gradf_logpdf(x, d = 0) for an EB/T spectrum x of shape (C, N, N/2+1)."""
        prec = prec or self.precision
        y = self._rfft2(self._lens(self._irfft2(self._apply(self.RT_c, x)), False, prec))
        h = self._mask_chain(y) if self.pixel_mask is not None else self._apply(self.W_data, y)
        z = self._rfft2(self._lens(self._irfft2(h), True, prec))
        return -(self._apply(self.R_c, z) + self._apply(self.Cf_inv, x))

    def b_vector(self, prec=None):
        """b = -gradf_logpdf(0, d) (wiener_filter.py:29-33)."""
        prec = prec or self.precision
        d = torch.stack([getattr(self.data, k) for k in self.data._matrix_names()])
        if self.pixel_mask is not None:
            rt_cn, bm_r = self._b_parts
            t = self._rfft2(self._irfft2(self._apply(rt_cn, d)) * self.pixel_mask)  # QU after Cn^-1 and m
            v = self._apply(bm_r, t)                                               # EB after B
            h = self._apply(self.RT_c, v)
        else:
            h = self._apply(self.RT_c, self._apply(self._bm_cn, d))
        z = self._rfft2(self._lens(self._irfft2(h), True, prec))
        return -self._apply(self.R_c, z)

    def dot(self, a, b):
        """fields.dot: Re sum conj(a) b w / N^2, float64, as a device scalar."""
        return torch.real(torch.sum(torch.conj(a) * b * self.weights)) / (self.N * self.N)

    # ------------------------------------------------------------ solve
    def solve(self, x0=None, rel_tol=None, tol=1e-1, maxiter=500, refine_every=0, check_every=1, history=None):
        """PCG with the reference recurrence; returns (x, iterations).  Stopping as wiener_filter.py:75-77
        (r.z < tol) unless ``rel_tol`` is given (||r|| / ||b||)."""
        b = self.b_vector()
        x = torch.zeros_like(b) if x0 is None else x0
        r = b - self.apply_A(x) if x0 is not None else b.clone()
        z = self._apply(self.P_inv, r)
        p = z.clone()
        res = self.dot(r, z)
        bnorm = torch.sqrt(self.dot(b, b))
        it = 0
        while it < maxiter:
            if it % check_every == 0:
                if rel_tol is None:
                    if not float(res) >= tol:
                        break
                else:
                    rn = float(torch.sqrt(torch.clamp(self.dot(r, r), min=0.0)) / bnorm)
                    if history is not None:
                        history.append(rn)
                    if rn < rel_tol:
                        break
            Ap = self.apply_A(p)
            alpha = res / self.dot(p, Ap)
            x = x + alpha * p
            it += 1
            if refine_every and it % refine_every == 0:
                r = b - self.apply_A(x, "f64")
            else:
                r = r - alpha * Ap
            z = self._apply(self.P_inv, r)
            res_new = self.dot(r, z)
            p = z + (res_new / res) * p
            res = res_new
        return x, it

    def to_field(self, x):
        """The solution as a reference-shaped field on the host."""
        return self.data.replace(**{k: x[i].cpu().numpy() for i, k in enumerate(self.data._matrix_names())})
