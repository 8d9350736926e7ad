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
                    n=10, scheme="reference", precision="f32"):
    """d logpdf / d phi for a Fourier phi: jax.grad(logpdf, argnums=1) of gradients.py:30-37, by hand.

    The data term's cotangent w.r.t. the lensed map is the ordinary partial
    derivative irfft2(eb2qu(B M Cn^-1 (d - M B L f)) * w / w_std), which the
    engine's reverse pass (the reference's custom VJP, lense_flow.py:23-46)
    turns into a Fourier delta-phi; the phi prior's custom VJP
    (statistics.py:199-209) adds -Cphi^-1 phi.  ``scheme="exact"`` uses the
    checkpointed reverse pass instead: the exact gradient of the discrete
    lens, without the reference scheme's RK4 discretisation gap.
    """
    fmap = map(eb2qu(unlensed_field))
    lensed_map = lense_flow(fmap, phi, n=n, precision=precision)
    resid = data - mask * beam * qu2eb(fourier(lensed_map))
    h = eb2qu(beam * mask * (pinv(noise_covariance) * resid))
    names = h._matrix_names()
    ratio = _weight_ratio(data.nside, resid.fourier_weights, getattr(h, names[0]))
    cot = map(h.replace(**{nm: getattr(h, nm) * ratio for nm in names}))
    _, dphi = lense_flow_backwards(lensed_map, phi, cot, n=n, direction=FORWARD_LENSE, precision=precision,
                                   scheme=scheme, field=fmap)
    prior = pinv(phi_covariance) * phi
    return dphi.replace(scalar_matrix=dphi.scalar_matrix - prior.scalar_matrix, fourier_weights=phi.fourier_weights,
                        basis=Basis.FOURIER, parametrization=Parametrization.T)


# ------------------------------------------------------------ mixed parametrisation
def _stack(field):
    """[1, C, N, N] float64 device tensor of a map-basis field's matrices."""
    return torch.stack([getattr(field, nm).to(torch.float64) for nm in field._matrix_names()]).unsqueeze(0)


def _unstack(like, t):
    return like.replace(**{nm: t[0, i] for i, nm in enumerate(like._matrix_names())})


@on_device
def mixing_jacobian_phi_component(mixed_field, phi, grad_f, mixing_d, n=10, precision="f32"):
    """gradients.py:63-85: the pullback of phi -> map(D^-1 qu2eb(fourier(L^-1(phi) map(eb2qu(f_mixed))))).

    phi is Fourier-shaped; the result is the Fourier delta-phi.  The
    pullbacks of ``map``, D^-1, ``qu2eb`` and ``fourier`` applied to the
    cotangent map(grad_f) compose to the cotangent map(eb2qu(D^-1
    fourier(map(grad_f)))) of the inverse-lensed map (JAX's irfft2 transpose
    w conj(rfft2(.)) / N^2 and rfft2 transpose N^2 irfft2(conj(.) / w) cancel),
    which the engine's reverse pass integrates with direction -1.
    """
    from .constants import INVERSE_LENSE
    mmap = map(eb2qu(mixed_field))
    unlensed = lense_flow(mmap, phi, n=n, direction=INVERSE_LENSE, precision=precision)
    cot = map(eb2qu(pinv(mixing_d) * fourier(map(grad_f))))
    _, dphi = lense_flow_backwards(unlensed, phi, cot, n=n, direction=INVERSE_LENSE, precision=precision)
    return dphi.replace(fourier_weights=phi.fourier_weights, basis=Basis.FOURIER, parametrization=Parametrization.T)


@on_device
def mixed_grad_phi_logpdf(mixed_field, mixed_phi, data, noise_covariance, phi_covariance, field_covariance, mask,
                          beam, mixing_d, mixing_g, n=10, precision="f32"):
    """d logpdf / d phi_mixed = G^-1 (grad_phi logpdf + J_phi^T grad_f logpdf) at the unmixed point (gradients.py:41-60).

    The reference composes ``unmix``, ``grad_phi_logpdf``, ``gradf_logpdf``
    and ``mixing_jacobian_phi_component``: five LenseFlow integrations and two
    reverse passes, with phi entering as map(phi) in unmix / gradf and as the
    Fourier phi in grad_phi / the Jacobian.  The two forms carry the same
    information when phi's DC and Nyquist columns are Hermitian
    (rfft2(irfft2(phi)) equals phi to 1e-12 relative), the usual case for a
    phi that came from a real map.  Then one set of derivative planes serves
    all four and the inverse lens of the mixed field and the forward lens of
    the unmixed field are run once and shared: two integrations, one adjoint
    integration and two reverse passes.  Otherwise each form gets its own
    planes and integrations, exactly as the reference composes them.
    """
    from . import engine
    from .constants import INVERSE_LENSE
    phi = pinv(mixing_g) * mixed_phi
    phif = phi.scalar_matrix.to(torch.complex128)
    mmap = map(eb2qu(mixed_field))
    ms = _stack(mmap)
    N, C = ms.shape[-1], ms.shape[1]
    plan = engine.get_plan(N, C, mmap.pix_width, precision, device=ms.device)
    phim = map(phi)
    drift = (fourier(phim).scalar_matrix - phif).abs().max()
    shared = bool(drift <= 1e-12 * phif.abs().max())
    planes_f = plan.phi_planes(phif.unsqueeze(0), check_det=True)
    planes_m = planes_f if shared else plan.phi_planes(phim.scalar_matrix.to(torch.float64).unsqueeze(0),
                                                       check_det=False)

    # unmix (map phi) and the Jacobian's inverse lens (Fourier phi)
    u_m = plan.lense_flow(ms, planes_m, n=n, direction=INVERSE_LENSE)
    u_f = u_m if shared else plan.lense_flow(ms, planes_f, n=n, direction=INVERSE_LENSE)
    field = pinv(mixing_d) * qu2eb(fourier(_unstack(mmap, u_m)))

    # forward lens of the unmixed field: grad_phi (Fourier phi) and gradf (map phi)
    fmap = map(eb2qu(field))
    fs = _stack(fmap)
    lensed_f = plan.lense_flow(fs, planes_f, n=n)
    lensed_m = lensed_f if shared else plan.lense_flow(fs, planes_m, n=n)

    def weighted_residual(lensed):
        resid = data - mask * beam * qu2eb(fourier(_unstack(fmap, lensed)))
        return resid, beam * mask * (pinv(noise_covariance) * resid)

    # grad_phi_logpdf's data term, then its prior
    resid, wres = weighted_residual(lensed_f)
    h = eb2qu(wres)
    names = h._matrix_names()
    ratio = _weight_ratio(data.nside, resid.fourier_weights, getattr(h, names[0]))
    cot = _stack(map(h.replace(**{nm: getattr(h, nm) * ratio for nm in names})))
    _, dphi_data = plan.lense_flow_vjp(lensed_f, cot, planes_f, n=n, direction=FORWARD_LENSE, phi_basis="fourier")
    grad_phi = dphi_data[0] - (pinv(phi_covariance) * phi).scalar_matrix

    # gradf_logpdf
    wres_m = wres if shared else weighted_residual(lensed_m)[1]
    back = plan.lense_flow(_stack(map(eb2qu(wres_m))), planes_m, n=n, adjoint=True)
    grad_f = qu2eb(fourier(_unstack(fmap, back))) - pinv(field_covariance) * qu2eb(fourier(fmap))

    # mixing Jacobian: reverse pass of the inverse lens
    cot_j = _stack(map(eb2qu(pinv(mixing_d) * fourier(map(grad_f)))))
    _, dphi_jac = plan.lense_flow_vjp(u_f, cot_j, planes_f, n=n, direction=INVERSE_LENSE, phi_basis="fourier")

    out = phi.replace(scalar_matrix=grad_phi + dphi_jac[0], fourier_weights=phi.fourier_weights,
                      basis=Basis.FOURIER, parametrization=Parametrization.T)
    return pinv(mixing_g) * out
