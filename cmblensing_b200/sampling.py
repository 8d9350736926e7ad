"""Simulation and the Gibbs/HMC steps around the lensing path, on the GPU engine.

Restates cmb_lensing/simulate.py:106-113 (Gaussian random fields from a
Fourier-diagonal covariance), the data model d = M B L(phi) f + n
(simulate.py:690-702), and sampling_ar.py:15-135 (gibbs_sample_f, the mass
matrix, the leapfrog integrator and the HMC step for the mixed phi).

Random draws: the reference uses jax.random, which is not available here;
these functions draw standard normals on the device with a torch generator
(``generator=``), or take the draws explicitly (``draws=``) so that a run can
be reproduced exactly -- the parity tests use the explicit form.
"""
from __future__ import annotations

import math

import torch

from ._device import device as _device, on_device
from .fields import FlatS0, _irfft2, _rfft2, dot, eb2qu, fourier, map, qu2eb
from .gradients import mixed_grad_phi_logpdf
from .lense_flow import lense_flow
from .matrix_operators import pinv
from .statistics import mixed_logpdf
from .wiener_filter import wiener_filter


def standard_normals(nside, generator=None, device=None):
    """Two independent (N, N/2+1) float64 standard normal arrays on the device."""
    dev = device if device is not None else (generator.device if generator is not None else _device())
    shape = (nside, nside // 2 + 1)
    a = torch.randn(shape, generator=generator, dtype=torch.float64, device=dev)
    b = torch.randn(shape, generator=generator, dtype=torch.float64, device=dev)
    return a, b


def field_from_normals(nside, covar_matrix, real_normals, imag_normals):
    """irfft2(sqrt(C/2) (a + i b), norm="ortho") -- simulate.py:106-113 with the draws given."""
    dev = covar_matrix.device if isinstance(covar_matrix, torch.Tensor) else _device()
    real_normals = torch.as_tensor(real_normals, dtype=torch.float64, device=dev)
    imag_normals = torch.as_tensor(imag_normals, dtype=torch.float64, device=dev)
    c = torch.as_tensor(covar_matrix, device=dev)
    spec = torch.sqrt(c.real / 2 if c.is_complex() else c / 2) * torch.complex(real_normals, imag_normals)
    return _irfft2(spec) * nside  # numpy's backward normalisation times N = ortho


def field_from_covar_single_key(nside, covar_matrix, generator=None, draws=None):
    """simulate.py:106-113: a real (N, N) Gaussian random field with Fourier covariance ``covar_matrix``."""
    dev = covar_matrix.device if isinstance(covar_matrix, torch.Tensor) and covar_matrix.is_cuda else None
    a, b = draws if draws is not None else standard_normals(nside, generator, dev)
    return field_from_normals(nside, covar_matrix, a, b)


@on_device
def simulate_data(field, phi, mask, beam, noise_covariance, generator=None, noise_draws=None, n=10):
    """d = M B L(phi) f + n, n ~ N(0, Cn) per component (simulate.py:690-702), in the EB (or T) Fourier basis."""
    nside = field.nside
    lensed = qu2eb(fourier(lense_flow(map(eb2qu(field)), map(phi), n=n)))
    names = lensed._matrix_names()
    cn = _diagonals(noise_covariance, names)
    noise = {}
    for i, nm in enumerate(names):
        d = noise_draws[i] if noise_draws is not None else None
        noise[nm] = _rfft2(field_from_covar_single_key(nside, cn[i], generator, d))
    return mask * beam * lensed + lensed.replace(**noise)


def _diagonals(op, names):
    """The per-component Fourier diagonals of a diagonal operator (T / EE, BB / TT, EE, BB)."""
    if len(names) == 1:
        return [op.scalar_matrix]
    if len(names) == 2:
        return [op.matrix_EE, op.matrix_BB]
    return [op.matrix_TT, op.matrix_EE, op.matrix_BB]


@on_device
def gibbs_sample_f(field_start, data_field, phi, field_covariance, noise_covariance, mask, beam, generator=None,
                   draws=None, n=10, maxiter=500, tol=1e-1):
    """sampling_ar.py:15-46: a constrained realisation f_sim + WF(d - (M B L f_sim + n_sim)).

    ``draws`` = ((a_f, b_f), (a_n, b_n)) fixes the field and noise normals;
    otherwise they come from ``generator``.  T fields, as in the reference
    (it reads ``args["field_covariance"].scalar_matrix``).
    """
    nside = data_field.nside
    fd, nd = draws if draws is not None else (None, None)
    new_field = field_start.replace(scalar_matrix=_rfft2(
        field_from_covar_single_key(nside, field_covariance.scalar_matrix, generator, fd)))
    new_noise = field_start.replace(scalar_matrix=_rfft2(
        field_from_covar_single_key(nside, noise_covariance.scalar_matrix, generator, nd)))
    lensed = qu2eb(fourier(lense_flow(map(eb2qu(new_field)), map(phi), n=n)))
    new_data = mask * beam * lensed + new_noise
    delta = wiener_filter.__wrapped__(field_start, phi, data_field - new_data, field_covariance, noise_covariance,
                                      mask, beam, n=n, maxiter=maxiter, tol=tol)
    return new_field + delta


def get_mass_matrix(cphi, nphi, mixing_g):
    """sampling_ar.py:65-66: G^-1 G^-1 (Cphi^-1 + Nphi^-1)."""
    return pinv(mixing_g) * pinv(mixing_g) * (pinv(cphi) + pinv(nphi))


@on_device
def symplectic_integrate(x0, p0, mixed_field, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                         mixing_d, mixing_g, mass_matrix, num_steps=30, step_size=0.01, n=10):
    """sampling_ar.py:104-135: leapfrog on the mixed phi (gradient of +logpdf); returns (delta H, x, p)."""
    def grad(x):
        return mixed_grad_phi_logpdf.__wrapped__(mixed_field, x, data, noise_covariance, phi_covariance,
                                                 field_covariance, mask, beam, mixing_d, mixing_g, n=n)

    def hamiltonian(x, p):
        lp = mixed_logpdf.__wrapped__(mixed_field, x, data, noise_covariance, phi_covariance, field_covariance,
                                      mask, beam, mixing_g, mixing_d, n=n)
        return lp - dot(p, (pinv(mass_matrix) * p) / 2)

    minv = pinv(mass_matrix)
    g = grad(x0)
    x, p = x0, p0
    for _ in range(num_steps):
        prev = g
        x = x - step_size * (minv * (p - 0.5 * step_size * g))
        g = grad(x)
        p = p - 0.5 * step_size * (g + prev)
    return float(hamiltonian(x, p) - hamiltonian(x0, p0)), x, p


@on_device
def hmc_step(x, always_accept, mass_matrix, mixed_field, data, noise_covariance, phi_covariance, field_covariance,
             mask, beam, mixing_d, mixing_g, generator=None, draws=None, num_steps=30, step_size=0.01, n=10):
    """sampling_ar.py:69-100: one HMC step for the mixed phi; returns (phi, delta H, accepted).

    ``draws`` = (a_p, b_p, log_u) fixes the momentum normals and log(uniform).
    The momentum is a T field with the mixed field's Fourier weights (the
    reference builds it as ``mixed_field.replace(scalar_matrix=...)``, which
    only a T-carrying field accepts).
    """
    nside = x.nside
    dev = x.scalar_matrix.device
    mass_matrix = mass_matrix.replace(scalar_matrix=torch.as_tensor(mass_matrix.scalar_matrix, device=dev))
    if draws is None:
        a, b = standard_normals(nside, generator, dev)
        log_u = math.log(float(torch.rand((), generator=generator, dtype=torch.float64, device=dev)))
    else:
        a, b, log_u = draws
    p = FlatS0(scalar_matrix=_rfft2(field_from_normals(nside, mass_matrix.scalar_matrix, a, b)), nside=nside,
               theta_pix=x.theta_pix, pix_width=x.pix_width, fourier_weights=mixed_field.fourier_weights)
    delta_h, x_test, _ = symplectic_integrate.__wrapped__(x, p, mixed_field, data, noise_covariance, phi_covariance,
                                                          field_covariance, mask, beam, mixing_d, mixing_g,
                                                          mass_matrix, num_steps=num_steps, step_size=step_size,
                                                          n=n)
    accept = bool(always_accept or (log_u < delta_h))
    return (x_test if accept else x), delta_h, accept
