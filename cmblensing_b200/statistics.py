"""logpdf of the lensed-CMB posterior (cmb_lensing/statistics.py:139-165) on the GPU engine."""
from __future__ import annotations

from ._device import on_device
from .fields import dot, eb2qu, fourier, map, qu2eb
from .lense_flow import lense_flow
from .matrix_operators import log_det, pinv


def _real(x):
    try:
        return x.real
    except AttributeError:
        return x


@on_device
def logpdf(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, n=10):
    """-1/2 [ |d - M B L(phi) f|^2_Cn + f^T Cf^-1 f + phi^T Cphi^-1 phi + 3 log-determinants ].

    ``field`` and ``data`` are EB (or T) Fourier fields, ``phi`` a Fourier
    FlatS0; the lensing runs on the CUDA engine with phi kept in Fourier space
    (derivatives from the rfft2 matrix, lense_flow.py:299-300).
    """
    logdets = log_det(phi_covariance) + log_det(noise_covariance) + log_det(field_covariance)
    prior_f = dot(field, pinv(field_covariance) * field)
    prior_phi = dot(phi, pinv(phi_covariance) * phi)
    lensed = qu2eb(fourier(lense_flow(map(eb2qu(field)), phi, n=n)))
    resid = data - mask * beam * lensed
    like = dot(resid, pinv(noise_covariance) * resid)
    return -_real(like + prior_f + prior_phi + logdets) / 2


@on_device
def mixed_logpdf(mixed_field, mixed_phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                 mixing_g, mixing_d, n=10):
    """statistics.py:168-181: logpdf at unmix(f_mixed, phi_mixed) minus Re log det G and Re log det D."""
    from .mixing import unmix
    field, phi = unmix.__wrapped__(mixed_field, mixed_phi, mixing_d, mixing_g, n=n)
    value = logpdf.__wrapped__(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, n=n)
    return value - _real(log_det(mixing_g)) - _real(log_det(mixing_d))
