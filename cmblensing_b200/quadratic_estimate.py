"""Quadratic-estimate noise N_phi (cmb_lensing/simulate.py:198-385) on the GPU.

``scalar_quadratic_estimate`` (T) and ``polar_quadratic_estimate`` (EB)
keep the reference's signatures and arithmetic: for each pair (i, j) of
x/y indices, products of inverse-transformed "legs" (spectra times
(i K_x)^a (i K_y)^b / |K|^c), transformed back, differentiated by d_i d_j,
and N_phi = 1 / sum_ij |.|.  Every leg of a call is an independent inverse
FFT, so they are gathered into one batch for the engine's float64 FFT
kernels (the polarization estimate has 16 non-zero Levi-Civita index sets
x 4 (i, j) x 6 legs); the K grid has no Nyquist flip, as the reference's
quadratic-estimate helpers have none.
"""
from __future__ import annotations

import itertools

import numpy as np
import torch

from ._device import device as _device
from .fields import _irfft2, _rfft2


def _t(x, dev):
    return torch.as_tensor(np.asarray(x) if not isinstance(x, torch.Tensor) else x, device=dev)


def _k_grid(N, pix_width, dev):
    kx = torch.as_tensor(2 * np.pi * np.fft.fftfreq(N, pix_width), device=dev)
    ky = torch.as_tensor(2 * np.pi * np.fft.rfftfreq(N, pix_width), device=dev)
    return torch.meshgrid(kx, ky, indexing="ij")


def _indices(length):
    """simulate.py:198-213: every 0/1 tuple of ``length`` (0 = x, 1 = y), grouped by the number of zeros."""
    out = []
    for n0 in range(length + 1):
        for zeros in itertools.combinations(range(length), n0):
            out.append(tuple(0 if i in zeros else 1 for i in range(length)))
    return out


def _safe_div(a, b):
    """a / b with NaN -> 0 (the reference's nan_to_num after each division by a vanishing spectrum)."""
    return torch.nan_to_num(a / b, nan=0.0)


class _Legs:
    """Collects leg spectra, inverse-transforms them in one batch, hands back the maps."""

    def __init__(self, N, pix_width, dev):
        self.KX, self.KY = _k_grid(N, pix_width, dev)
        self.lap = self.KX ** 2 + self.KY ** 2
        self.items = []

    def add(self, spec, encapsulated, isolated):
        """qe_leg (simulate.py:272-302): (i KX)^nx (i KY)^ny F / |K|^len(isolated)."""
        idx = list(encapsulated) + list(isolated)
        ny = sum(idx)
        nx = len(idx) - ny
        f = torch.nan_to_num(spec.to(torch.complex128), nan=0.0)
        if nx or ny:
            mult = (1j * self.KX) ** nx * (1j * self.KY) ** ny
            f = torch.nan_to_num(mult * f / torch.sqrt(self.lap ** len(isolated)), nan=0.0)
        self.items.append(f)
        return len(self.items) - 1

    def maps(self):
        return _irfft2(torch.stack(self.items))


def _finish(internal, pix_width, pairs):
    """1 / sum_ij |d_i d_j rfft2(internal_ij)| with 1/0 -> 0 (simulate.py:305-315, :318-331)."""
    N = internal.shape[-1]
    KX, KY = _k_grid(N, pix_width, internal.device)
    K = (KX, KY)
    spec = _rfft2(internal)
    total = torch.zeros_like(KX)
    for s, (i, j) in enumerate(pairs):
        total = total + torch.abs(-(K[i] * K[j]) * spec[s])
    return torch.nan_to_num(1 / total, nan=0.0, posinf=0.0, neginf=0.0)


def scalar_quadratic_estimate(cn_tt, cf_tt, cfl_tt, m_tt, b_tt, pix_width):
    """simulate.py:305-315 (legs: simulate.py:357-367): the T quadratic-estimate noise, float64 on the GPU."""
    dev = cf_tt.device if isinstance(cf_tt, torch.Tensor) and cf_tt.is_cuda else _device()
    cn, cf, cfl, m, b = (_t(x, dev) for x in (cn_tt, cf_tt, cfl_tt, m_tt, b_tt))
    N = cf.shape[0]
    tf = m * b
    sigma = tf ** 2 * cfl + cn
    a1, a0, a2 = _safe_div(tf ** 2 * cf ** 2, sigma), _safe_div(tf ** 2, sigma), _safe_div(tf ** 2 * cf, sigma)
    legs = _Legs(N, pix_width, dev)
    pairs = _indices(2)
    ids = [(legs.add(a1, (i, j), ()), legs.add(a0, (), ()), legs.add(a2, (i,), ()), legs.add(a2, (j,), ()))
           for i, j in pairs]
    x = legs.maps()
    internal = torch.stack([x[p] * x[q] + x[r] * x[s] for p, q, r, s in ids])
    return _finish(internal, pix_width, pairs)


def polar_quadratic_estimate(cf_ee, cf_bb, cfl_ee, cfl_bb, cn_ee, cn_bb, mask_ee, mask_bb, beam_ee, beam_bb,
                             pix_width):
    """simulate.py:318-354 (legs: simulate.py:370-385): the EB quadratic-estimate noise, float64 on the GPU."""
    dev = cf_ee.device if isinstance(cf_ee, torch.Tensor) and cf_ee.is_cuda else _device()
    cfe, cfb, cle, clb, cne, cnb, me, mb, be, bb = (_t(x, dev) for x in (cf_ee, cf_bb, cfl_ee, cfl_bb, cn_ee,
                                                                           cn_bb, mask_ee, mask_bb, beam_ee,
                                                                           beam_bb))
    N = cfe.shape[0]
    tf2e, tf2b = (me * be) ** 2, (mb * bb) ** 2
    se, sb = tf2e * cle + cne, tf2b * clb + cnb
    e2, e1, e0 = _safe_div(tf2e * cfe ** 2, se), _safe_div(tf2e * cfe, se), _safe_div(tf2e, se)
    b2, b1, b0 = _safe_div(tf2b * cfb ** 2, sb), _safe_div(tf2b * cfb, sb), _safe_div(tf2b, sb)
    # Levi-Civita epsilon[m, p, 2] for m, p in {0, 1}: +1 at (0, 1), -1 at (1, 0), 0 on the diagonal
    eps = lambda u, v: 0 if u == v else (1 if (u, v) == (0, 1) else -1)
    legs = _Legs(N, pix_width, dev)
    pairs = _indices(2)
    terms = []  # per (i, j): list of (weight, leg ids of the three products)
    for i, j in pairs:
        tj = []
        for (k, l, m, n, p, q) in _indices(6):
            w = 4 * eps(m, p) * eps(n, q)
            if w == 0:
                continue
            klmn, klpq = (k, l, m, n), (k, l, p, q)
            tj.append((w, legs.add(e2, (i, j), klmn), legs.add(b0, (), klpq), legs.add(e1, (i,), klmn),
                       legs.add(b1, (j,), klpq), legs.add(e0, (), klmn), legs.add(b2, (i, j), klpq)))
        terms.append(tj)
    x = legs.maps()
    internal = torch.stack([sum(w * (x[a] * x[b] - 2 * x[c] * x[d] + x[e] * x[f]) for w, a, b, c, d, e, f in tj)
                            for tj in terms])
    return _finish(internal, pix_width, pairs)
