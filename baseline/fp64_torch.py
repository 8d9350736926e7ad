"""Plain float64 GPU comparator: the reference's LenseFlow op sequence restated with torch.

This is NOT the reference (jax is not installed on this machine or the GPU
box).  It restates cmb_lensing/lense_flow.py:289-415 and util.py:103-199
op for op in float64 with torch.fft (cuFFT) on batched maps, computing only
the two derivatives the standard term uses (what XLA's dead-code
elimination would keep).  It exists only as the "plain FP64 GPU path"
baseline for bench.py.
"""
import math

import torch


def _kgrid(N, pix_width, device):
    kx = 2 * math.pi * torch.fft.fftfreq(N, pix_width, dtype=torch.float64, device=device)
    ky = 2 * math.pi * torch.fft.rfftfreq(N, pix_width, dtype=torch.float64, device=device)
    ky[-1] = -ky[-1]
    return kx[:, None], ky[None, :]


def _irf(X, N):
    return torch.fft.irfft2(X, s=(N, N))


def phi_derivs(phi, pix_width):
    N = phi.shape[-1]
    KX, KY = _kgrid(N, pix_width, phi.device)
    F = torch.fft.rfft2(phi)
    return (_irf(1j * KX * F, N), _irf(1j * KY * F, N), _irf(-(KX ** 2) * F, N), _irf(-(KX * KY) * F, N),
            _irf(-(KY ** 2) * F, N))


def standard_term(y, d, t, pix_width):
    phi_x, phi_y, phi_xx, phi_xy, phi_yy = d
    N = y.shape[-1]
    KX, KY = _kgrid(N, pix_width, y.device)
    F = torch.fft.rfft2(y)
    fx, fy = _irf(1j * KX * F, N), _irf(1j * KY * F, N)
    mxx, mxy, myy = 1 + t * phi_xx, t * phi_xy, 1 + t * phi_yy
    inv = 1.0 / (mxx * myy - mxy * mxy + 1e-12)
    ixx, ixy, iyy = myy * inv, -mxy * inv, mxx * inv
    vx = fx * ixx + fy * ixy
    vy = fy * iyy + fx * ixy
    return phi_x * vx + phi_y * vy


def lense_flow_fp64(f, phi, pix_width, n=7):
    """Forward lens of f [B, C, N, N] with phi [B, N, N], float64, per component as the reference does."""
    out = torch.empty_like(f)
    h = 1.0 / n
    for c in range(f.shape[1]):
        d = phi_derivs(phi, pix_width)  # recomputed per component (lense_flow.py:290-302)
        y = f[:, c]
        for i in range(n):
            t = i * h
            k1 = standard_term(y, d, t, pix_width)
            k2 = standard_term(y + h / 2 * k1, d, t + h / 2, pix_width)
            k3 = standard_term(y + h / 2 * k2, d, t + h / 2, pix_width)
            k4 = standard_term(y + h * k3, d, t + h, pix_width)
            y = y + h * (k1 + 2 * k2 + 2 * k3 + k4) / 6
        out[:, c] = y
    return out
