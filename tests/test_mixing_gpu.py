"""GPU parity of mix, unmix, mixing_jacobian_phi_component and mixed_grad_phi_logpdf against the oracle.

Inputs: the reference's golden T and QU sets (256^2, 2.5', DC/Nyquist
Fourier weight 1) with their mixing diagonals D and G; n = 7.  Tolerances
follow the other inference tests: FP32 lensing gives ~1e-7 relative error
per integration, so the gradients agree with the float64 oracle to 2e-5
relative L2 and the mixed fields to 1e-5.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import lenseflow_ref as R
from test_inference_gpu import _Mod, _sets

pytestmark = pytest.mark.gpu
N = 256


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _mixing(which, mod):
    m = load_golden("mix.npz")
    w = R.get_fourier_weights((N, N))
    if which == "I":
        D = mod.DiagonalScalar(scalar_matrix=m["d_t"], fourier_weights=w)
    else:
        D = mod.DiagonalEB(matrix_EE=m["d_ee"], matrix_BB=m["d_bb"], fourier_weights=w)
    return D, mod.DiagonalScalar(scalar_matrix=m["g"], fourier_weights=w)


def _both(which):
    _, S = _sets(which, _Mod())
    _, So = _sets(which, R)
    return S, So, _mixing(which, _Mod()), _mixing(which, R)


@pytest.mark.parametrize("which", ["I", "P"])
def test_mix_unmix(torch_cuda, which):
    from cmblensing_b200.mixing import mix, unmix
    S, So, (D, G), (Do, Go) = _both(which)
    fm, pm = mix(S["field"], S["phi"], D, G, n=7)
    fmo, pmo = R.mix(So["field"], So["phi"], Do, Go, n=7)
    for nm in fmo._matrix_names():
        assert rel_l2(getattr(fm, nm), getattr(fmo, nm)) < 1e-5
    assert rel_l2(pm.scalar_matrix, pmo.scalar_matrix) < 1e-14
    f, phi = unmix(fm, pm, D, G, n=7)
    fo, phio = R.unmix(fmo, pmo, Do, Go, n=7)
    for nm in fo._matrix_names():
        assert rel_l2(getattr(f, nm), getattr(fo, nm)) < 1e-5
    assert rel_l2(phi.scalar_matrix, phio.scalar_matrix) < 1e-14


@pytest.mark.parametrize("which", ["I", "P"])
def test_mixing_jacobian(torch_cuda, which):
    from cmblensing_b200.gradients import mixing_jacobian_phi_component
    S, So, (D, G), (Do, Go) = _both(which)
    fmo, _ = R.mix(So["field"], So["phi"], Do, Go, n=7)
    grad_f = R.gradf_logpdf(So["field"], So["phi"], So["data"], So["Cf"], So["Cn"], So["M"], So["B"], n=7)
    ref = R.mixing_jacobian_phi_component(fmo, So["phi"], grad_f, Do, n=7)
    mod = _Mod()
    fm = (mod.FlatS0 if which == "I" else mod.FlatS2)(**{nm: getattr(fmo, nm) for nm in fmo._matrix_names()},
                                                      fourier_weights=fmo.fourier_weights)
    gf = fm.replace(**{nm: getattr(grad_f, nm) for nm in grad_f._matrix_names()})
    out = mixing_jacobian_phi_component(fm, S["phi"], gf, D, n=7)
    assert rel_l2(out.scalar_matrix, ref) < 2e-5


@pytest.mark.parametrize("which", ["I", "P"])
def test_mixed_grad_phi_logpdf(torch_cuda, which):
    """The engine's shared-work pipeline against the oracle's restatement of gradients.py:41-60."""
    from cmblensing_b200.gradients import mixed_grad_phi_logpdf
    from cmblensing_b200.mixing import mix
    S, So, (D, G), (Do, Go) = _both(which)
    fmo, pmo = R.mix(So["field"], So["phi"], Do, Go, n=7)
    ref = R.mixed_grad_phi_logpdf(fmo, pmo, So["data"], So["Cn"], So["Cphi"], So["Cf"], So["M"], So["B"], Do, Go,
                                  n=7)
    fm, pm = mix(S["field"], S["phi"], D, G, n=7)
    out = mixed_grad_phi_logpdf(fm, pm, S["data"], S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], D, G, n=7)
    assert rel_l2(out.scalar_matrix, ref) < 2e-5
    # the Julia golden, to the oracle's own bound
    m = load_golden("mix.npz")
    r, c = m["idx"]
    assert rel_l2(out.scalar_matrix[r, c], m["mixed_grad_phi_" + which]) < 1e-3


def test_mixed_grad_phi_matches_reference_composition(torch_cuda):
    """Shared and unshared lens passes against the engine's own unmix / grad_phi / gradf / Jacobian chain.

    The golden phi is Hermitian on its DC column, so the shared branch runs;
    its derivative planes differ from the map(phi) ones by float64 rounding
    only (a few FP32 last-bit flips), so the two agree to FP32 rounding.  A
    phi whose DC column is not Hermitian takes the unshared branch, which
    launches exactly the reference composition's kernels on the same inputs.
    """
    from cmblensing_b200.gradients import (grad_phi_logpdf, gradf_logpdf, mixed_grad_phi_logpdf,
                                           mixing_jacobian_phi_component)
    from cmblensing_b200.matrix_operators import pinv
    from cmblensing_b200.mixing import mix, unmix
    S, _, (D, G), _ = _both("P")
    fm, pm = mix(S["field"], S["phi"], D, G, n=7)
    rng = np.random.default_rng(11)
    skew = pm.scalar_matrix.copy()
    skew[1:N // 2, 0] += 1e-3 * np.abs(skew[1:N // 2, 0]) * rng.standard_normal(N // 2 - 1)
    for phi_m, tol in ((pm, 1e-6), (pm.replace(scalar_matrix=skew), 1e-12)):
        args = (S["data"], S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"])
        fused = mixed_grad_phi_logpdf(fm, phi_m, *args, D, G, n=7)
        f, phi = unmix(fm, phi_m, D, G, n=7)
        gp = grad_phi_logpdf(f, phi, *args, n=7)
        gf = gradf_logpdf(f, phi, S["data"], S["Cf"], S["Cn"], S["M"], S["B"], n=7)
        jac = mixing_jacobian_phi_component(fm, phi, gf, D, n=7)
        ref = (pinv(G) * gp.replace(scalar_matrix=gp.scalar_matrix + jac.scalar_matrix)).scalar_matrix
        assert rel_l2(fused.scalar_matrix, ref) < tol
