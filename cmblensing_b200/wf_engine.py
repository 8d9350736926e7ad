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

The per-mode products run in one fused kernel each (lf_modes_apply: real
float64 matrices, blocks that are zero everywhere skipped), the FFTs on the
engine's float64 kernels, and the maps between the FFTs and the lens are
float32 for the FP32 operator (float64 for the FP64 operator of the
true-residual refinement).  The CG keeps every vector and scalar on the
device; a problem that has converged is masked on the device (alpha =
beta = 0), so a block of iterations needs no host decision and is captured
once as a CUDA graph and replayed: the host synchronises once per block,
not once per iteration.  Optional true-residual replacement every
``refine_every`` iterations uses the FP64 engine for b - A x.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native as nat
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


def _nonzero_mask(W):
    """Bit i*C+j set where block (i, j) of the per-mode operator W ((B,)C,C,N,H) is not identically zero."""
    Wb = W if W.dim() == 5 else W.unsqueeze(0)
    C = Wb.shape[1]
    nz = (Wb != 0).flatten(3).any(dim=3).any(dim=0).cpu().tolist()
    return sum(1 << (i * C + j) for i in range(C) for j in range(C) if nz[i][j])


class DeviceWienerFilter:
    """Wiener filters of a batch of problems (same N, components and pixel size), resident on the GPU.

    ``problems`` is a list of dicts with keys phi, data, Cf, Cn, M, B
    (reference-shaped containers, host or device).  One application of A
    lenses the whole batch in one engine launch sequence; the CG scalars are
    per problem, and a problem that has converged keeps its iterate while the
    others continue.  ``DeviceWienerFilter(phi, data, Cf, Cn, M, B)`` builds a
    batch of one.
    """

    def __init__(self, phi=None, data=None, field_covariance=None, noise_covariance=None, mask=None, beam=None,
                 n=10, precision="f32", problems=None):
        if problems is None:
            problems = [dict(phi=phi, data=data, Cf=field_covariance, Cn=noise_covariance, M=mask, B=beam)]
        dev = device()
        self.dev = dev
        self.n = n
        self.precision = precision
        self.batch = len(problems)
        d0 = problems[0]["data"]
        self.C = C = _ncomp(d0)
        self.N = N = d0.nside
        self.pw = d0.pix_width
        self.theta = d0.theta_pix
        self.datas, Rt, Wd, Bc, Cfi, Pinv, masks, Wb, Wn, bparts, phis, weights = [], [], [], [], [], [], [], [], [], [], [], []
        for prob in problems:
            phi_, data, Cf, Cn, B = [to_device(prob[k], dev) for k in ("phi", "data", "Cf", "Cn", "B")]
            if (_ncomp(data), data.nside, data.theta_pix) != (C, N, self.theta):
                raise ValueError("a batch of Wiener filters must share N, components and pixel size")
            mask = prob["M"]
            first = getattr(data, data._matrix_names()[0])
            self.datas.append(data)
            weights.append(torch.as_tensor(np.real(np.asarray(data.fourier_weights)), device=dev))
            R = self._rotation(C, N, data.theta_pix, first)
            RT = R.transpose(0, 1).contiguous()
            Cn_inv = _op_matrix(pinv(Cn), C, first)
            Bm = _op_matrix(B, C, first)
            Cfi.append(_op_matrix(pinv(Cf), C, first))
            if isinstance(mask, PixelMask):
                masks.append(to_device(mask, dev).mask_map)
                Mm = _op_matrix(mask.diagonal_like(B), C, first)
                Wb.append(_mm(RT, _mm(Bm, R)))
                Wn.append(_mm(RT, _mm(Cn_inv, R)))
                bparts.append((_mm(RT, Cn_inv), _mm(Bm, R)))
            else:
                masks.append(None)
                Mm = _op_matrix(mask, C, first)
                Wd.append(_mm(RT, _mm(_mm(Bm, _mm(Mm, _mm(Cn_inv, _mm(Mm, Bm)))), R)))
                Bc.append(_mm(Bm, _mm(Mm, Cn_inv)))
            P = _op_matrix(pinv(Cf), C, first) + _mm(Bm, _mm(Mm, _mm(Cn_inv, _mm(Mm, Bm))))
            Pinv.append(self._invert(P))
            phis.append(to_map(phi_).scalar_matrix.to(torch.float64))
        kinds = {m is None for m in masks}
        if len(kinds) != 1:
            raise ValueError("a batch mixes map-space and Fourier-diagonal masks")
        # per-mode operators as real float64 (C, C, N, H) (shared) or (B, C, C, N, H) (per problem)
        st = lambda lst: torch.stack(lst).to(torch.float64).contiguous()
        self.R_c = R.to(torch.float64).contiguous()          # identical for the batch (same N, pixel size)
        self.RT_c = RT.to(torch.float64).contiguous()
        self.Cf_inv = st(Cfi)
        self.P_inv = st(Pinv)
        self.weights = torch.stack(weights)[:, None, None, :]  # (B, 1, 1, N/2+1)
        self.pixel_mask = None
        if masks[0] is not None:
            pm = torch.stack(masks)[:, None]                     # (B, 1, N, N)
            self.pixel_mask = {"f64": pm.to(torch.float64), "f32": pm.to(torch.float32)}
            self.W_b, self.W_n = st(Wb), st(Wn)
            self._b_rt_cn = st([b[0] for b in bparts])
            self._b_bm_r = st([b[1] for b in bparts])
        else:
            self.W_data, self._bm_cn = st(Wd), st(Bc)
        self.d = torch.stack([torch.stack([getattr(dd, k) for k in dd._matrix_names()]) for dd in self.datas])
        self.phimap = torch.stack(phis)
        self.plan = engine.get_plan(N, C, self.pw, precision, device=dev)
        self.planes = engine.cached_phi_planes(self.plan, self.phimap)
        self.fft = engine.get_plan(N, 1, self.pw, "f64", device=dev)
        self._plan64 = None
        self._lib = self.plan._lib
        # which C x C blocks of every per-mode operator are not identically zero (found once, here)
        self._nonzero = {}
        for W in [self.R_c, self.RT_c, self.Cf_inv, self.P_inv] + (
                [self.W_b, self.W_n, self._b_rt_cn, self._b_bm_r] if self.pixel_mask is not None
                else [self.W_data, self._bm_cn]):
            self._nonzero[(W.data_ptr(), tuple(W.shape))] = _nonzero_mask(W)
        self.graph_blocks = 0  # CG blocks replayed from a captured graph in the last solve

    # ----------------------------------------------------------- pieces
    @staticmethod
    def _rotation(C, N, theta, like):
        """Per-mode qu2eb rotation (util.py:152-161), identity on T."""
        R = torch.zeros((C, C, N, N // 2 + 1), dtype=torch.float64, device=like.device)
        if C == 1:
            R[0, 0] = 1.0
            return R
        c2a, s2a = _eb_angle(N, theta, like)
        o = C - 2
        if C == 3:
            R[0, 0] = 1.0
        R[o, o], R[o, o + 1] = -c2a, -s2a
        R[o + 1, o], R[o + 1, o + 1] = s2a, -c2a
        return R

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
            sc = rec(a - b * rd * c)
            out[0, 0], out[0, 1], out[1, 0], out[1, 1] = sc, -sc * b * rd, -rd * c * sc, rd + rd * c * sc * b * rd
            out[2, 2] = rec(P[2, 2])
        return out

    def _apply(self, W, X, scale=1.0, Y=None, yscale=0.0):
        """scale * (W X) + yscale * Y per mode: W (C,C,N,H) shared or (B,C,C,N,H) per problem (real float64);
        X, Y (B,C,N,H) complex128.  One fused kernel (lf_modes_apply)."""
        B, C = X.shape[0], X.shape[1]
        X = X.contiguous()
        out = torch.empty(X.shape, dtype=torch.complex128, device=X.device)
        nz = self._nonzero[(W.data_ptr(), tuple(W.shape))]
        st = ctypes.c_void_p(torch.cuda.current_stream(X.device).cuda_stream)
        nat.check(self._lib.lf_modes_apply(ctypes.c_void_p(W.data_ptr()), int(W.dim() == 5), nz,
                                           ctypes.c_void_p(X.data_ptr()),
                                           ctypes.c_void_p(Y.contiguous().data_ptr()) if Y is not None else None,
                                           ctypes.c_void_p(out.data_ptr()), B, C, X.shape[2] * X.shape[3],
                                           float(scale), float(yscale), st), "lf_modes_apply")
        return out

    def _irfft2(self, X, prec="f64"):
        """irfft2 of (B, C, N, H) spectra into float64 maps, or float32 maps for the FP32 operator."""
        B, C = X.shape[:2]
        dt = torch.float32 if prec == "f32" else torch.float64
        return self.fft.irfft2(X.reshape(B * C, self.N, self.N // 2 + 1), out_dtype=dt).reshape(B, C, self.N,
                                                                                                 self.N)

    def _rfft2(self, X):
        B, C = X.shape[:2]
        return self.fft.rfft2(X.reshape(B * C, self.N, self.N)).reshape(B, C, self.N, self.N // 2 + 1)

    def _lens(self, q, adjoint, prec):
        if prec == self.precision:
            plan, planes = self.plan, self.planes
        else:
            if self._plan64 is None:
                self._plan64 = engine.get_plan(self.N, self.C, self.pw, prec, device=self.dev)
                self._planes64 = engine.cached_phi_planes(self._plan64, self.phimap)
            plan, planes = self._plan64, self._planes64
        return plan.lense_flow(q, planes, n=self.n, adjoint=adjoint)

    def _mask_chain(self, y, prec):
        """QU spectra -> W y through the map-space mask: B, m, Cn^-1, m, B (maps in the operator's precision)."""
        m = self.pixel_mask[prec]
        t = self._apply(self.W_b, y)
        t = self._rfft2(self._irfft2(t, prec) * m)
        t = self._apply(self.W_n, t)
        t = self._rfft2(self._irfft2(t, prec) * m)
        return self._apply(self.W_b, t)

    def apply_A(self, x, prec=None):
        """A x = gradf_logpdf(x, d = 0) for EB/T spectra x of shape (B, C, N, N/2+1) (or (C, N, N/2+1))."""
        single = x.dim() == 3
        if single:
            x = x.unsqueeze(0)
        prec = prec or self.precision
        y = self._rfft2(self._lens(self._irfft2(self._apply(self.RT_c, x), prec), False, prec))
        h = self._mask_chain(y, prec) if self.pixel_mask is not None else self._apply(self.W_data, y)
        z = self._rfft2(self._lens(self._irfft2(h, prec), True, prec))
        out = self._apply(self.Cf_inv, x, -1.0, self._apply(self.R_c, z), -1.0)  # -(R z + Cf^-1 x)
        return out[0] if single else out

    def b_vector(self, prec=None):
        """b = -gradf_logpdf(0, d) (wiener_filter.py:29-33), (B, C, N, N/2+1)."""
        prec = prec or self.precision
        if self.pixel_mask is not None:
            t = self._rfft2(self._irfft2(self._apply(self._b_rt_cn, self.d)) * self.pixel_mask["f64"])
            h = self._apply(self.RT_c, self._apply(self._b_bm_r, t))
        else:
            h = self._apply(self.RT_c, self._apply(self._bm_cn, self.d))
        z = self._rfft2(self._lens(self._irfft2(h, prec), True, prec))
        return self._apply(self.R_c, z, -1.0)

    def dot(self, a, b):
        """fields.dot per problem: Re sum conj(a) b w / N^2, float64 device tensor of shape (B,)."""
        return torch.real(torch.sum(torch.conj(a) * b * self.weights, dim=(1, 2, 3))) / (self.N * self.N)

    # ------------------------------------------------------------ solve
    def _iteration(self, S, refine):
        """One PCG iteration of the reference recurrence on the device state S (updated in place).

        Inactive problems get alpha = beta = 0 (their iterate stays), and the
        stopping rule is evaluated on the device at the end of the iteration,
        so a block of iterations needs no host decision."""
        bc = lambda v: v[:, None, None, None]
        active = S["active"]
        Ap = self.apply_A(S["p"])
        pAp = self.dot(S["p"], Ap)
        alpha = torch.where(active, S["res"] / torch.where(pAp != 0, pAp, torch.ones_like(pAp)),
                            torch.zeros_like(pAp))
        S["x"].add_(bc(alpha) * S["p"])
        S["iters"].add_(active.to(torch.int64))
        if refine:  # true residual with the FP64 engine (residual replacement)
            S["r"].copy_(torch.where(bc(active), S["b"] - self.apply_A(S["x"], "f64"), S["r"]))
        else:
            S["r"].sub_(bc(alpha) * Ap)
        z = self._apply(self.P_inv, S["r"])
        res_new = self.dot(S["r"], z)
        beta = torch.where(active, res_new / torch.where(S["res"] != 0, S["res"], torch.ones_like(res_new)),
                           torch.zeros_like(res_new))
        S["p"].copy_(z + bc(beta) * S["p"])
        S["res"].copy_(torch.where(active, res_new, S["res"]))
        self._update_active(S)

    def _update_active(self, S):
        """Stopping rule per problem (wiener_filter.py:75-77: r.z < tol; or ||r|| / ||b|| < rel_tol)."""
        if S["rel_tol"] is None:
            S["active"].logical_and_(S["res"] >= S["tol"])
        else:
            rn = torch.sqrt(torch.clamp(self.dot(S["r"], S["r"]), min=0.0)) / S["bnorm"]
            S["rn"].copy_(rn)
            S["active"].logical_and_(~(rn < S["rel_tol"]))

    def solve(self, x0=None, rel_tol=None, tol=1e-1, maxiter=500, refine_every=0, check_every=10, history=None,
              use_graphs=True):
        """PCG with the reference recurrence for every problem; returns (x, iterations) for a batch of one,
        else (x [B, C, N, N/2+1], iterations per problem).  Stopping per problem as wiener_filter.py:75-77
        (r.z < tol) unless ``rel_tol`` is given (||r|| / ||b||).

        Iterations run in blocks of ``refine_every`` (else ``check_every``);
        the host reads whether any problem is still active once per block.
        With ``use_graphs`` the first block runs eagerly (kernel attributes,
        the FP64 refinement plan), the second is captured as a CUDA graph, and
        every later full block replays it.  The iteration counts per problem
        equal those of a per-iteration check (the stopping rule is applied on
        the device every iteration); ``history`` (per-iteration ||r||/||b||)
        forces eager blocks of one iteration."""
        b = self.b_vector()
        x = torch.zeros_like(b) if x0 is None else (x0 if x0.dim() == 4 else x0.unsqueeze(0)).clone()
        r = b - self.apply_A(x) if x0 is not None else b.clone()
        z = self._apply(self.P_inv, r)
        S = {"b": b, "x": x, "r": r, "p": z.clone(), "res": self.dot(r, z),
             "bnorm": torch.sqrt(self.dot(b, b)), "rel_tol": rel_tol, "tol": tol,
             "active": torch.ones(self.batch, dtype=torch.bool, device=self.dev),
             "iters": torch.zeros(self.batch, dtype=torch.int64, device=self.dev),
             "rn": torch.zeros(self.batch, dtype=torch.float64, device=self.dev)}
        self._update_active(S)
        k = int(refine_every) if refine_every else max(1, int(check_every))
        if history is not None:
            k, use_graphs = 1, False
        it = 0
        graph = None
        self.graph_blocks = 0
        while it < maxiter:
            if history is not None and S["rel_tol"] is not None:
                history.append(S["rn"].cpu().numpy())
            if not bool(S["active"].any()):  # one host synchronisation per block
                break
            engine.check_timeouts("Wiener filter")
            m = min(k, maxiter - it)
            refine_at = [j for j in range(m) if refine_every and (it + j + 1) % refine_every == 0]
            full = m == k and it % k == 0
            if use_graphs and full and it > 0:
                if graph is None:  # no device-wide synchronisation: other threads may be capturing too
                    def block():
                        for j in range(m):
                            self._iteration(S, j in refine_at)
                    graph = engine.capture_graph(block)
                graph.replay()
                self.graph_blocks += 1
            else:
                for j in range(m):
                    self._iteration(S, j in refine_at)
            it += m
        its = S["iters"].cpu().tolist()
        engine.check_timeouts("Wiener filter")
        x = S["x"]
        if self.batch == 1:
            return x[0], its[0]
        return x, its

    def to_field(self, x, i=0):
        """Solution ``i`` (or the only one) as a reference-shaped field on the host."""
        xi = x if x.dim() == 3 else x[i]
        data = self.datas[i]
        return data.replace(**{k: xi[j].cpu().numpy() for j, k in enumerate(data._matrix_names())})
