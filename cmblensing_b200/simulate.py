"""Seeded synthetic inputs with the workloads' spectra (host, numpy float64).

Gaussian random fields follow the reference's recipe
(cmb_lensing/simulate.py:71-113): a Fourier-diagonal covariance
C(k) = C_l(|k|) / d^2 (d = pixel width in radians), a field
irfft2(sqrt(C/2) (a + i b), norm="ortho") with a, b ~ N(0, 1), and the
l = 0 mode zeroed.  Each field is then rescaled to the stated rms.

phi spectrum: C_l ~ 1 / [l^2 (l+1)^2 (1 + (l/60)^2)], normalised to a
2.5 arcmin rms deflection.  The literal form with (1 + (l/60)^-2) has an
l^-4 tail that makes det(I + t grad grad phi) negative at these pixel
sizes, so LenseFlow is singular for it; ``spectrum="literal"`` keeps it
available with the deflection normalisation given by the caller.
"""
from __future__ import annotations

import math

import numpy as np

ARCMIN = math.pi / (180.0 * 60.0)


def ell_grid(nside, theta_pix):
    """|l| on the (N, N/2+1) rfft2 grid (util.py:163-179)."""
    d = theta_pix * ARCMIN
    lx = 2 * np.pi * np.fft.rfftfreq(nside, d)
    ly = 2 * np.pi * np.fft.fftfreq(nside, d)
    lx, ly = np.meshgrid(lx, ly)
    return np.sqrt(lx ** 2 + ly ** 2), d


def _grf(cl, nside, theta_pix, rng):
    ell, d = ell_grid(nside, theta_pix)
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.where(ell > 0, cl(np.where(ell > 0, ell, 1.0)), 0.0) / d ** 2
    a = rng.standard_normal(c.shape)
    b = rng.standard_normal(c.shape)
    return np.fft.irfft2(np.sqrt(c / 2) * (a + 1j * b), s=(nside, nside), norm="ortho")


SPECTRA = {
    "TT": lambda l: l ** -2.0 * np.exp(-(l / 2500.0) ** 2),
    "EE": lambda l: l ** -2.0 * np.exp(-(l / 2000.0) ** 2),
}
RMS_UK = {"TT": 100.0, "EE": 5.0}


def gaussian_field(nside, theta_pix, kind="TT", seed=0, rms=None):
    """A real (N, N) map with C_l of ``kind`` ("TT" or "EE") scaled to ``rms`` (default 100 / 5 uK)."""
    rng = np.random.default_rng(seed)
    f = _grf(SPECTRA[kind], nside, theta_pix, rng)
    target = RMS_UK[kind] if rms is None else rms
    return f * (target / np.sqrt(np.mean(f ** 2)))


def deflection_rms(phi, theta_pix):
    """rms of |grad phi| in radians."""
    n = phi.shape[0]
    d = theta_pix * ARCMIN
    kx = 2 * np.pi * np.fft.fftfreq(n, d)[:, None]
    ky = 2 * np.pi * np.fft.rfftfreq(n, d)[None, :]
    F = np.fft.rfft2(phi)
    gx = np.fft.irfft2(1j * kx * F, s=(n, n))
    gy = np.fft.irfft2(1j * ky * F, s=(n, n))
    return float(np.sqrt(np.mean(gx ** 2 + gy ** 2)))


def phi_spectrum(spectrum="wellposed"):
    if spectrum == "literal":
        return lambda l: 1.0 / (l ** 2 * (l + 1) ** 2 * (1 + (l / 60.0) ** -2))
    return lambda l: 1.0 / (l ** 2 * (l + 1) ** 2 * (1 + (l / 60.0) ** 2))


def gaussian_phi(nside, theta_pix, seed=0, deflection_arcmin=2.5, spectrum="wellposed"):
    """Lensing potential map (N, N) with rms deflection ``deflection_arcmin``."""
    rng = np.random.default_rng(seed)
    phi = _grf(phi_spectrum(spectrum), nside, theta_pix, rng)
    return phi * (deflection_arcmin * ARCMIN / deflection_rms(phi, theta_pix))


def min_magnification_det(phi, theta_pix):
    """min over pixels and t in [0,1] of det(I + t grad grad phi) (float64, host)."""
    n = phi.shape[0]
    d = theta_pix * ARCMIN
    kx = 2 * np.pi * np.fft.fftfreq(n, d)[:, None]
    ky = 2 * np.pi * np.fft.rfftfreq(n, d).copy()
    ky[-1] = -ky[-1]
    ky = ky[None, :]
    F = np.fft.rfft2(phi)
    a = np.fft.irfft2(-kx * kx * F, s=(n, n))
    b = np.fft.irfft2(-kx * ky * F, s=(n, n))
    c = np.fft.irfft2(-ky * ky * F, s=(n, n))
    q = a * c - b * b
    lin = a + c
    best = np.minimum(1.0, 1.0 + lin + q)
    with np.errstate(divide="ignore", invalid="ignore"):
        ts = np.where(q > 0, -lin / (2 * q), -1.0)
    inside = (ts > 0) & (ts < 1)
    best = np.where(inside, np.minimum(best, 1.0 + ts * lin + ts * ts * q), best)
    return float(best.min())


def qu_from_e(e_map, theta_pix):
    """Q, U maps of a pure-E field (B = 0) with the reference's EB->QU rotation (util.py:140-149)."""
    n = e_map.shape[0]
    d = theta_pix * ARCMIN
    lx = 2 * np.pi * np.fft.rfftfreq(n, d)
    ly = 2 * np.pi * np.fft.fftfreq(n, d)
    lx, ly = np.meshgrid(lx, ly)
    lx[: n // 2 + 1, -1] *= -1
    a = np.arctan2(lx, ly)
    E = np.fft.rfft2(e_map)
    q = np.fft.irfft2(-E * np.cos(2 * a), s=(n, n))
    u = np.fft.irfft2(-E * np.sin(2 * a), s=(n, n))
    return q, u


def lens_batch(nside, theta_pix, batch, ncomp, seed0=0):
    """(fields [B, C, N, N], phis [B, N, N]) float64 for C = 1 (T), 2 (QU) or 3 (TQU)."""
    f = np.empty((batch, ncomp, nside, nside))
    phis = np.empty((batch, nside, nside))
    for i in range(batch):
        phis[i] = gaussian_phi(nside, theta_pix, seed=1000 + seed0 + i)
        if ncomp in (1, 3):
            f[i, 0] = gaussian_field(nside, theta_pix, "TT", seed=2000 + seed0 + i)
        if ncomp in (2, 3):
            e = gaussian_field(nside, theta_pix, "EE", seed=2500 + seed0 + i)
            q, u = qu_from_e(e, theta_pix)
            f[i, ncomp - 2] = q
            f[i, ncomp - 1] = u
    return f, phis


# ------------------------------------------------- inference problems
def _cl_grid(cl, nside, theta_pix):
    ell, d = ell_grid(nside, theta_pix)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(ell > 0, cl(np.where(ell > 0, ell, 1.0)), 0.0) / d ** 2


def beam_grid(nside, theta_pix, fwhm_arcmin):
    """B(l) = exp(-l^2 sigma^2 / 2), sigma = FWHM / sqrt(8 ln 2), zero at l = 0 (simulate.py:133-138)."""
    ell, _ = ell_grid(nside, theta_pix)
    sig = fwhm_arcmin * ARCMIN / math.sqrt(8 * math.log(2))
    b = np.exp(-(ell ** 2) * sig ** 2 / 2)
    b[0, 0] = 0.0
    return b


def hole_mask(nside, theta_pix, nholes=30, rmin=5.0, rmax=20.0, apod=10.0, seed=5000):
    """Pixel mask with ``nholes`` circular holes (radius rmin..rmax arcmin) and a cosine taper of ``apod`` arcmin."""
    rng = np.random.default_rng(seed)
    size = nside * theta_pix
    y, x = np.meshgrid(np.arange(nside) * theta_pix, np.arange(nside) * theta_pix, indexing="ij")
    m = np.ones((nside, nside))
    for _ in range(nholes):
        cy, cx = rng.uniform(0, size, 2)
        r = rng.uniform(rmin, rmax)
        dy = np.minimum(np.abs(y - cy), size - np.abs(y - cy))  # periodic flat sky
        dx = np.minimum(np.abs(x - cx), size - np.abs(x - cx))
        d = np.sqrt(dx ** 2 + dy ** 2)
        w = np.where(d <= r, 0.0, np.where(d >= r + apod, 1.0, 0.5 * (1 - np.cos(np.pi * (d - r) / apod))))
        m *= w
    return m


def inference_problem(nside, theta_pix, beam_fwhm=3.0, noise_t=10.0, noise_p=14.0, seed=0, bb_fraction=0.0):
    """Host arrays of a lensed-CMB inference problem in the reference's units and layouts.

    Returns a dict with the unlensed fields ``t, e, b`` and the potential
    ``phi`` as unnormalised rfft2 arrays, noise realisations ``n_t, n_e, n_b``
    (white, ``noise_*`` uK-arcmin), and the Fourier-diagonal ``cf_tt, cf_ee,
    cf_bb, cn_t, cn_p, cphi, beam``.  Covariances are C_l / d^2
    (simulate.py:71-97) scaled by the factors the fields were rescaled by.
    The caller forms the data d = B L(phi) f + n with the lensing operator.
    The simulated B is zero; ``bb_fraction`` sets the prior C_BB to that
    fraction of C_EE (with C_BB = 0 the reference's pinv leaves B modes with
    no prior, and a masked Wiener filter is then nearly singular).
    """
    rng_seed = seed
    f_t = gaussian_field(nside, theta_pix, "TT", seed=2000 + rng_seed)
    f_e = gaussian_field(nside, theta_pix, "EE", seed=2500 + rng_seed)
    phi = gaussian_phi(nside, theta_pix, seed=1000 + rng_seed)
    # covariances with the normalisations the fields were rescaled by
    def scaled_cov(kind, fmap, seedv):
        raw = _grf(SPECTRA[kind], nside, theta_pix, np.random.default_rng(seedv))
        s = (RMS_UK[kind] / np.sqrt(np.mean(raw ** 2))) ** 2
        return _cl_grid(SPECTRA[kind], nside, theta_pix) * s
    cf_tt = scaled_cov("TT", f_t, 2000 + rng_seed)
    cf_ee = scaled_cov("EE", f_e, 2500 + rng_seed)
    raw_phi = _grf(phi_spectrum(), nside, theta_pix, np.random.default_rng(1000 + rng_seed))
    sphi = (2.5 * ARCMIN / deflection_rms(raw_phi, theta_pix)) ** 2
    cphi = _cl_grid(phi_spectrum(), nside, theta_pix) * sphi
    shape = cf_tt.shape
    out = dict(t=np.fft.rfft2(f_t), e=np.fft.rfft2(f_e), b=np.zeros(shape, complex), phi=np.fft.rfft2(phi),
               cf_tt=cf_tt, cf_ee=cf_ee, cf_bb=bb_fraction * cf_ee, cphi=cphi,
               cn_t=np.full(shape, (noise_t / theta_pix) ** 2), cn_p=np.full(shape, (noise_p / theta_pix) ** 2),
               beam=beam_grid(nside, theta_pix, beam_fwhm), nside=nside, theta_pix=theta_pix)
    rng = np.random.default_rng(3000 + rng_seed)
    out["n_t"] = np.fft.rfft2(rng.standard_normal((nside, nside)) * noise_t / theta_pix)
    out["n_e"] = np.fft.rfft2(rng.standard_normal((nside, nside)) * noise_p / theta_pix)
    out["n_b"] = np.fft.rfft2(rng.standard_normal((nside, nside)) * noise_p / theta_pix)
    return out
