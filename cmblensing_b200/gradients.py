"""Gradients of logpdf (cmb_lensing/gradients.py:13-37) on the GPU engine."""
from __future__ import annotations

import numpy as np

from .constants import Basis, FORWARD_LENSE, Parametrization
from ._device import on_device
from .fields import eb2qu, fourier, get_fourier_weights, map, qu2eb
from .lense_flow import lense_flow, lense_flow_backwards
from .matrix_operators import pinv

try:
    import torch
except Exception:  # pragma: no cover
    torch = None


@on_device
def gradf_logpdf(field, phi, data, field_covariance, noise_covariance, mask, beam, n=10, precision="f32"):
    """d logpdf / d f = L^dag B M Cn^-1 (d - M B L f) - Cf^-1 f, in the EB Fourier basis.

    Two LenseFlow passes (forward, then adjoint) on the engine; phi enters
    through its map (gradients.py:17), and the prior term uses the field
    round-tripped through map space as the reference does.
    """
    fmap = map(eb2qu(field))
    phimap = map(phi)
    lensed = qu2eb(fourier(lense_flow(fmap, phimap, n=n, precision=precision)))
    weighted = beam * mask * pinv(noise_covariance) * (data - mask * beam * lensed)
    back = lense_flow(map(eb2qu(weighted)), phimap, n=n, adjoint=True, precision=precision)
    return qu2eb(fourier(back)) - pinv(field_covariance) * qu2eb(fourier(fmap))


def _weight_ratio(nside, weights, like):
    """w / w_std, with w_std = (1, 2, ..., 2, 1) the column weights implied by irfft2."""
    r = np.real(np.asarray(weights if not (torch is not None and isinstance(weights, torch.Tensor))
                           else weights.cpu().numpy()) / get_fourier_weights((nside, nside)))
    if torch is not None and isinstance(like, torch.Tensor):
        return torch.as_tensor(r, device=like.device)
    return r


@on_device
def grad_phi_logpdf(unlensed_field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                    n=10):
    """d logpdf / d phi for a Fourier phi: jax.grad(logpdf, argnums=1) of gradients.py:30-37, by hand.

    The data term's cotangent w.r.t. the lensed map is the ordinary partial
    derivative irfft2(eb2qu(B M Cn^-1 (d - M B L f)) * w / w_std), which the
    engine's reverse pass (the reference's custom VJP, lense_flow.py:23-46)
    turns into a Fourier delta-phi; the phi prior's custom VJP
    (statistics.py:199-209) adds -Cphi^-1 phi.
    """
    fmap = map(eb2qu(unlensed_field))
    lensed_map = lense_flow(fmap, phi, n=n)
    resid = data - mask * beam * qu2eb(fourier(lensed_map))
    h = eb2qu(beam * mask * (pinv(noise_covariance) * resid))
    names = h._matrix_names()
    ratio = _weight_ratio(data.nside, resid.fourier_weights, getattr(h, names[0]))
    cot = map(h.replace(**{nm: getattr(h, nm) * ratio for nm in names}))
    _, dphi = lense_flow_backwards(lensed_map, phi, cot, n=n, direction=FORWARD_LENSE)
    prior = pinv(phi_covariance) * phi
    return dphi.replace(scalar_matrix=dphi.scalar_matrix - prior.scalar_matrix, fourier_weights=phi.fourier_weights,
                        basis=Basis.FOURIER, parametrization=Parametrization.T)
