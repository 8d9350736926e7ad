"""The oracle's restatement of the checkpointed exact reverse pass, pinned on the CPU.

``lensing_operator_gradients_exact`` has no counterpart in the reference (it
restates the engine's extension lf_lense_flow_vjp_ckpt), so it is pinned by
what it claims to be: the gradient of the discrete lens.  Central finite
differences with a small step (1e-6 of the rms) agree with it to rounding
level (1e-6 here), for a map phi and for a Fourier phi (complex coefficients,
torch's dL/dRe + i dL/dIm convention = delta-phi * w / N^2); its delta-f equals
the reference scheme's (the adjoint lens is already the exact transpose); and
its delta-phi differs from the reference scheme's only by the RK4
discretisation gap of the latter.
"""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import lenseflow_ref as R

N, THETA, NSTEPS = 32, 3.0, 4


def _inputs(C, seed=3):
    from cmblensing_b200.simulate import lens_batch
    f, phis = lens_batch(N, THETA, 1, C, seed0=seed)
    return f[0], phis[0]


def _tqu(arr):
    z = np.zeros_like(arr[0])
    return {1: lambda: (arr[0], z, z), 2: lambda: (z, arr[0], arr[1]), 3: lambda: tuple(arr)}[len(arr)]()


@pytest.mark.parametrize("C,direction", [(1, 1), (2, -1), (3, 1)])
def test_exact_scheme_is_the_discrete_gradient_map_phi(C, direction):
    pw = R.pix_width_of(THETA)
    f, phi = _inputs(C)
    g = np.random.default_rng(1).standard_normal(f.shape)
    res = R.lensing_operator_gradients_exact(phi, pw, _tqu(f), _tqu(g), direction, NSTEPS)

    def loss(p):
        return sum(np.sum(R.primal_lense_flow(f[c], p, pw, NSTEPS, direction, False) * g[c]) for c in range(C))

    rms = np.sqrt(np.mean(phi ** 2))
    rng = np.random.default_rng(2)
    for _ in range(2):
        v = rng.standard_normal(phi.shape)
        eps = 1e-6 * rms
        fd = (loss(phi + eps * v) - loss(phi - eps * v)) / (2 * eps)
        assert abs(np.sum(res[6] * v) - fd) / abs(fd) < 1e-6
    # delta-f: the reference scheme's (exact transpose), lensed output: the forward lens
    lz = [R.primal_lense_flow(f[c], phi, pw, NSTEPS, direction, False) for c in range(C)]
    ref = R.get_lensing_operator_gradients(phi, pw, _tqu(lz), _tqu(g), -direction, NSTEPS)
    for a, b in zip(res[3:6], ref[3:6]):
        if np.any(b):
            assert rel_l2(a, b) < 1e-12
    for a, b in zip(res[0:3], _tqu(lz)):
        if np.any(b):
            assert rel_l2(a, b) < 1e-13
    # the reference scheme's delta-phi carries the RK4 gap: close, not equal
    gap = rel_l2(ref[6], res[6])
    assert 1e-8 < gap < 1e-2


def test_exact_scheme_fourier_phi_convention():
    pw = R.pix_width_of(THETA)
    f, phi = _inputs(2, seed=5)
    phif = np.fft.rfft2(phi)
    g = np.random.default_rng(4).standard_normal(f.shape)
    res = R.lensing_operator_gradients_exact(phif, pw, _tqu(f), _tqu(g), 1, NSTEPS)
    w = R.get_fourier_weights((N, N)).real
    grad = res[6] * w / N ** 2

    def loss(p):
        return sum(np.sum(R.primal_lense_flow(f[c], p, pw, NSTEPS, 1, False) * g[c]) for c in range(2))

    for k in [(3, 5), (10, 7), (20, 2)]:
        e = 1e-7 * np.abs(phif).max()
        vals = []
        for d in (e, -e, 1j * e, -1j * e):
            p = phif.copy()
            p[k] += d
            vals.append(loss(p))
        gre = (vals[0] - vals[1]) / (2 * e)
        gim = (vals[2] - vals[3]) / (2 * e)
        assert abs(grad[k].real - gre) / abs(gre) < 1e-5, (k, grad[k], gre, gim)
        assert abs(grad[k].imag - gim) / abs(gim) < 1e-5, (k, grad[k], gre, gim)
