"""MAP joint estimate of (f, phi) (cmb_lensing/map_joint.py:19-98) on the GPU engine.

``map_joint(data_set, num_steps=30, constant_step=False)`` keeps the
reference's loop: Wiener-filter f at the current phi, mix with G = 1, take
the mixed phi gradient and step phi <- phi + alpha H^-1 grad with
H = Cphi^-1 + Nphi^-1.  The reference picks alpha with scipy's BFGS on
-logpdf(alpha), one lens pair per evaluation, one evaluation at a time.
Here the default line search evaluates -logpdf at a set of alphas in one
batched engine call (every candidate's inverse and forward lens run as one
batch) and refines around the best candidate with a second batch and a
parabolic step; ``line_search="bfgs"`` runs the reference's scipy search on
the engine instead.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from . import engine
from ._device import on_device
from .constants import INVERSE_LENSE
from .fields import FlatS0, _irfft2, eb2qu, fourier, get_fourier_weights, map, qu2eb
from .gradients import mixed_grad_phi_logpdf
from .matrix_operators import DiagonalScalar, log_det, pinv
from .mixing import mix
from .statistics import logpdf
from .wiener_filter import wiener_filter


@dataclasses.dataclass
class DataSet:
    """The members of dataset.py:14-98 that the MAP and sampling loops read (T, EB or TEB operators)."""
    data: object = None
    noise_covariance: object = None
    mixing_d: object = None
    field_covariance: object = None
    phi_covariance: object = None
    quadratic_estimate: object = None
    mask: object = None
    beam: object = None
    mixing_g: object = None
    fid_r: float = 0.2
    fid_a_phi: float = 1.0


DataSetT = DataSetEB = DataSetTEB = DataSet


def get_scalar_identity(op):
    """matrix_operators.py:159-170: the identity DiagonalScalar shaped like ``op``."""
    shape = (op.nside, op.nside // 2 + 1)
    like = getattr(op, op._matrix_names()[0])
    ones = (torch.ones(shape, dtype=torch.complex128, device=like.device) if isinstance(like, torch.Tensor)
            else np.ones(shape, dtype=np.complex128))
    return DiagonalScalar(fourier_weights=get_fourier_weights(shape), nside=op.nside, theta_pix=op.theta_pix,
                          pix_width=op.pix_width, scalar_matrix=ones)


def zero_scalar_field_like(field):
    """fields.py:123-133: a zero Fourier T field with the field's geometry."""
    shape = (field.nside, field.nside // 2 + 1)
    like = getattr(field, field._matrix_names()[0])
    zeros = (torch.zeros(shape, dtype=torch.complex128, device=like.device) if isinstance(like, torch.Tensor)
             else np.zeros(shape, dtype=np.complex128))
    return FlatS0(fourier_weights=get_fourier_weights(shape), nside=field.nside, theta_pix=field.theta_pix,
                  pix_width=field.pix_width, scalar_matrix=zeros)


def phi_gradient_hessian(phi_covariance, quadratic_estimate):
    """map_joint.py:72-77: Cphi^-1 + Nphi^-1."""
    return pinv(phi_covariance) + pinv(quadratic_estimate)


def _dot_k(f1, f2):
    """dot (fields.py:137-142) per leading index of [K, N, N/2+1] matrices: Re sum conj(a) b w / N^2."""
    s = 0.0
    for nm in f1._matrix_names():
        a, b = getattr(f1, nm), getattr(f2, nm)
        w = torch.as_tensor(f1.fourier_weights, device=a.device)
        s = s + torch.real(torch.sum(torch.conj(a) * b * w, dim=(-2, -1))) / f1.nside ** 2
    return s


def _stack(field):
    return torch.stack([getattr(field, nm).to(torch.float64) for nm in field._matrix_names()], dim=-3)


def _unstack(like, t):
    return like.replace(**{nm: t[..., i, :, :] for i, nm in enumerate(like._matrix_names())})


@on_device
def neg_logpdf_along(alphas, grad_phi, mixed_field, mixed_phi, data, beam, mask, field_covariance, phi_covariance,
                     noise_covariance, mixing_d, mixing_g, hessian, n=10, precision="f32"):
    """-logpdf at unmix(f_mixed, phi_m + alpha H grad) for every alpha (map_joint.py:79-98), as one batch.

    The K candidates' inverse lenses (unmix, with map(phi)) run as one
    engine call over K maps, and so do their forward lenses (logpdf, with
    the Fourier phi); priors, residuals and log-determinants follow
    statistics.py:139-165 per candidate.  Returns a float64 tensor [K].
    """
    dev = mixed_phi.scalar_matrix.device
    a = torch.as_tensor(np.asarray(alphas, dtype=np.float64), device=dev).reshape(-1, 1, 1)
    K = a.shape[0]
    step = (hessian * grad_phi).scalar_matrix
    phi_k = pinv(mixing_g).scalar_matrix * (mixed_phi.scalar_matrix.unsqueeze(0) + a * step.unsqueeze(0))
    phi = mixed_phi.replace(scalar_matrix=phi_k)
    mmap = map(eb2qu(mixed_field))
    ms = _stack(mmap)
    C, N = ms.shape[0], ms.shape[-1]
    plan = engine.get_plan(N, C, mmap.pix_width, precision, device=dev)
    # unmix: inverse lens of the mixed field by each candidate's map(phi)
    planes_m = plan.phi_planes(_irfft2(phi_k).to(torch.float64), check_det=True)
    u = plan.lense_flow(ms.unsqueeze(0).expand(K, C, N, N).contiguous(), planes_m, n=n, direction=INVERSE_LENSE)
    field = pinv(mixing_d) * qu2eb(fourier(_unstack(mmap, u)))
    # logpdf at (field_k, phi_k), phi in the Fourier basis
    fmap = map(eb2qu(field))
    planes_f = plan.phi_planes(phi_k.to(torch.complex128), check_det=True)
    lensed = plan.lense_flow(_stack(fmap).contiguous(), planes_f, n=n)
    resid = data - mask * beam * qu2eb(fourier(_unstack(fmap, lensed)))
    like = _dot_k(resid, pinv(noise_covariance) * resid)
    prior_f = _dot_k(field, pinv(field_covariance) * field)
    prior_phi = _dot_k(phi, pinv(phi_covariance) * phi)
    logdets = torch.real(torch.as_tensor(log_det(phi_covariance) + log_det(noise_covariance)
                                         + log_det(field_covariance), device=dev))
    return (like + prior_f + prior_phi + logdets) / 2


def batched_line_search(evaluate, coarse=(0.25, 0.5, 1.0, 2.0, 4.0, 8.0), fine=7, max_extend=3):
    """Minimise ``evaluate(alphas) -> values`` over alpha > 0 with a few batched evaluations.

    1. the ``coarse`` set (extended upwards by factors of 8 while its largest
       alpha is best, at most ``max_extend`` times);
    2. ``fine`` points spanning the best coarse alpha's neighbours;
    3. the vertex of the parabola through the best fine point and its
       neighbours, evaluated once.
    Returns (alpha, value) of the best point evaluated.
    """
    a = np.asarray(coarse, dtype=np.float64)
    v = np.asarray(evaluate(a), dtype=np.float64)
    seen_a, seen_v = list(a), list(v)
    for _ in range(max_extend):
        if int(np.argmin(v)) != len(a) - 1:
            break
        a = a[-1] * np.asarray([2.0, 4.0, 8.0])
        v = np.asarray(evaluate(a), dtype=np.float64)
        seen_a += list(a)
        seen_v += list(v)
    order = np.argsort(seen_a)
    sa, sv = np.asarray(seen_a)[order], np.asarray(seen_v)[order]
    b = int(np.argmin(sv))
    lo = sa[b - 1] if b > 0 else 0.0
    hi = sa[b + 1] if b + 1 < len(sa) else 2.0 * sa[b]
    fa = np.linspace(lo, hi, fine + 2)[1:-1]
    fv = np.asarray(evaluate(fa), dtype=np.float64)
    xa = np.concatenate([sa, fa])
    xv = np.concatenate([sv, fv])
    order = np.argsort(xa)
    xa, xv = xa[order], xv[order]
    b = int(np.argmin(xv))
    if 0 < b < len(xa) - 1:
        x0, x1, x2 = xa[b - 1], xa[b], xa[b + 1]
        y0, y1, y2 = xv[b - 1], xv[b], xv[b + 1]
        den = (x0 - x1) * (x0 - x2) * (x1 - x2)
        A = (x2 * (y1 - y0) + x1 * (y0 - y2) + x0 * (y2 - y1)) / den
        B = (x2 * x2 * (y0 - y1) + x1 * x1 * (y2 - y0) + x0 * x0 * (y1 - y2)) / den
        if A > 0:
            xv_ = -B / (2 * A)
            if x0 < xv_ < x2:
                yv_ = float(np.asarray(evaluate(np.asarray([xv_])))[0])
                if yv_ < xv[b]:
                    return float(xv_), yv_
    return float(xa[b]), float(xv[b])


def map_joint(data_set, num_steps=30, constant_step=False, n=10, line_search="batched", wf_maxiter=500, wf_tol=1e-1,
              history=None):
    """map_joint.py:19-67: alternate Wiener-filter f-steps and preconditioned phi-steps; returns (f, phi).

    ``line_search``: "batched" (candidates evaluated as one engine batch,
    ``batched_line_search``) or "bfgs" (the reference's scipy BFGS from
    alpha = 1, one engine evaluation per call).  ``history`` (a list)
    receives (alpha, -logpdf at the step taken) per step.
    """
    from ._device import device as _dev, to_device, to_host
    ds = data_set
    data = ds.data
    host = not (isinstance(getattr(data, data._matrix_names()[0]), torch.Tensor)
                and getattr(data, data._matrix_names()[0]).is_cuda)
    dev = _dev()
    put = lambda o: to_device(o, dev)
    data, Cn, D, Cf, Cphi, QE, M, B = (put(o) for o in (ds.data, ds.noise_covariance, ds.mixing_d,
                                                       ds.field_covariance, ds.phi_covariance,
                                                       ds.quadratic_estimate, ds.mask, ds.beam))
    G = get_scalar_identity(D)  # the MAP estimate does not depend on G
    field = data * 0
    phi = zero_scalar_field_like(data)
    hessian = pinv(phi_gradient_hessian(Cphi, QE))
    alpha = 1.0
    for _ in range(num_steps):
        field = wiener_filter.__wrapped__(field, phi, data, Cf, Cn, M, B, n=n, maxiter=wf_maxiter, tol=wf_tol)
        mixed_field, mixed_phi = mix.__wrapped__(field, phi, D, G, n=n)
        grad = mixed_grad_phi_logpdf.__wrapped__(mixed_field, mixed_phi, data, Cn, Cphi, Cf, M, B, D, G, n=n)

        def evaluate(alphas):
            return neg_logpdf_along.__wrapped__(alphas, grad, mixed_field, mixed_phi, data, B, M, Cf, Cphi, Cn, D,
                                                G, hessian, n=n).cpu().numpy()

        value = None
        if not constant_step:
            if line_search == "bfgs":
                from scipy.optimize import minimize
                res = minimize(lambda a: float(evaluate(np.atleast_1d(a)[:1])[0]), 1.0, method="BFGS")
                alpha, value = float(res.x[0]), float(res.fun)
            else:
                alpha, value = batched_line_search(evaluate)
        if history is not None:
            history.append((alpha, value))
        phi = phi + alpha * (hessian * grad)
    if host:
        return to_host(field), to_host(phi)
    return field, phi
