"""Lensed Wiener filter by preconditioned CG (cmb_lensing/wiener_filter.py:11-104) on the GPU engine.

``wiener_filter(field, phi, data, Cf, Cn, M, B)`` keeps the reference's
signature and defaults (absolute stop r.z < 0.1, 500 iterations, n = 10
RK4 steps).  The operator A f = gradf_logpdf(f, d = 0) applies one forward
and one adjoint LenseFlow on the engine (FP32 by default); all inner
products are float64 reductions on the device.

Extensions used by the precision workload (not in the reference):
``rel_tol`` stops on ||r|| / ||b|| (norms from ``dot``) instead of r.z, and
``refine_every = k`` replaces the recurrence residual by the true residual
b - A x computed with the FP64 engine every k iterations (residual
replacement), so the FP32 operator's rounding does not limit the attainable
accuracy.
"""
from __future__ import annotations

import math

from ._device import on_device
from .fields import dot
from .gradients import gradf_logpdf
from .matrix_operators import PixelMask, pinv


def get_b_vector(phi, data, field_covariance, noise_covariance, mask, beam, n=10, precision="f32"):
    """wiener_filter.py:29-33: b = -gradf(0, d)."""
    return gradf_logpdf.__wrapped__(data * 0, phi, data, field_covariance, noise_covariance, mask, beam, n=n,
                                    precision=precision) * -1


def hessian_logpdf_preconditioner(field_covariance, beam, mask, noise_covariance):
    """wiener_filter.py:36-43: Cf^-1 + B M Cn^-1 M B (Fourier-diagonal).

    A map-space ``PixelMask`` enters through its Fourier-diagonal stand-in
    sqrt(mean(m^2)) (the preconditioner must stay diagonal).
    """
    if isinstance(mask, PixelMask):
        mask = mask.diagonal_like(beam)
    return pinv(field_covariance) + beam * mask * pinv(noise_covariance) * mask * beam


def _scalar(x):
    return float(x)


def conjugate_gradient(x0, data, phi, mask, beam, noise_covariance, field_covariance, b_vector, preconditioner,
                       maxiter=500, tol=1e-1, n=10, rel_tol=None, refine_every=0, precision="f32", history=None):
    """wiener_filter.py:52-104: the reference PCG recurrence; returns (x, iterations)."""

    def apply_A(f, prec):
        return gradf_logpdf.__wrapped__(f, phi, f * 0, field_covariance, noise_covariance, mask, beam, n=n,
                                        precision=prec)

    pinv_p = pinv(preconditioner)
    x = x0
    r = b_vector - apply_A(x0, precision)
    z = pinv_p * r
    p = z
    res = _scalar(dot(r, z))
    bnorm = math.sqrt(max(_scalar(dot(b_vector, b_vector)), 1e-300))
    it = 0
    while it < maxiter:
        if rel_tol is None:
            if not res >= tol:
                break
        else:
            rn = math.sqrt(max(_scalar(dot(r, r)), 0.0)) / bnorm
            if history is not None:
                history.append(rn)
            if rn < rel_tol:
                break
        Ap = apply_A(p, precision)
        alpha = res / _scalar(dot(p, Ap))
        x = x + alpha * p
        it += 1
        if refine_every and it % refine_every == 0:
            r = b_vector - apply_A(x, "f64")  # true residual with the FP64 engine
        else:
            r = r - alpha * Ap
        z = pinv_p * r
        res_new = _scalar(dot(r, z))
        p = z + (res_new / res) * p
        res = res_new
    return x, it


@on_device
def wiener_filter(field, phi, data, field_covariance, noise_covariance, mask, beam, n=10, maxiter=500, tol=1e-1,
                  rel_tol=None, refine_every=0, precision="f32", return_iterations=False):
    """wiener_filter.py:11-26."""
    b = get_b_vector(phi, data, field_covariance, noise_covariance, mask, beam, n=n, precision=precision)
    P = hessian_logpdf_preconditioner(field_covariance, beam, mask, noise_covariance)
    x, it = conjugate_gradient(field, data, phi, mask, beam, noise_covariance, field_covariance, b, P,
                               maxiter=maxiter, tol=tol, n=n, rel_tol=rel_tol, refine_every=refine_every,
                               precision=precision)
    if return_iterations:
        wiener_filter.last_iterations = it
    return x
