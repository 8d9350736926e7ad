"""Mixed parametrisation of (f, phi) (cmb_lensing/mixing.py:8-36) on the GPU engine.

``mix`` maps an unlensed EB/T Fourier field and a Fourier phi to
(qu2eb(fourier(L(phi) map(eb2qu(D f)))), G phi); ``unmix`` inverts it with
the inverse LenseFlow.  D and G are the reference's Fourier-diagonal mixing
operators.  Both keep the reference's signature; ``n`` (10 in the
reference, which hard-codes the LenseFlow default) and ``precision`` are
exposed as keywords.
"""
from __future__ import annotations

from ._device import on_device
from .constants import INVERSE_LENSE
from .fields import eb2qu, fourier, map, qu2eb
from .lense_flow import lense_flow
from .matrix_operators import pinv


@on_device
def mix(field, phi, mixing_d, mixing_g, n=10, precision="f32"):
    """mixing.py:8-20."""
    df = map(eb2qu(mixing_d * field))
    mixed_field = qu2eb(fourier(lense_flow(df, map(phi), n=n, precision=precision)))
    return mixed_field, mixing_g * phi


@on_device
def unmix(mixed_field, mixed_phi, mixing_d, mixing_g, n=10, precision="f32"):
    """mixing.py:23-36."""
    phi = pinv(mixing_g) * mixed_phi
    mmap = map(eb2qu(mixed_field))
    field = qu2eb(fourier(lense_flow(mmap, map(phi), n=n, direction=INVERSE_LENSE, precision=precision)))
    return pinv(mixing_d) * field, phi
