"""GPU parity of the simulation and sampling steps (simulate.py:106-113, sampling_ar.py:15-135) against the oracle.

Random draws are passed explicitly, so each device result is compared with
the float64 oracle on identical normals; the generator path is checked
statistically.  Inputs: the reference's golden T and QU sets (256^2, 2.5',
DC/Nyquist Fourier weight 1), n = 7 RK4 steps.  Tolerances: float64 FFTs
agree to 1e-12; anything that lenses in FP32 to 2e-5 relative L2 (as the
gradient tests); logpdf differences (delta H) to 1e-8 of |logpdf|.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import lenseflow_ref as R
from test_inference_gpu import _Mod, _sets
from test_mixing_gpu import _mixing

pytestmark = pytest.mark.gpu
N = 256


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _normals(seed, nside=N):
    rng = np.random.default_rng(seed)
    shape = (nside, nside // 2 + 1)
    return rng.standard_normal(shape), rng.standard_normal(shape)


def test_field_from_normals_matches_oracle(torch_cuda):
    from cmblensing_b200.sampling import field_from_normals
    g = load_golden("infer_I.npz")
    a, b = _normals(1)
    out = field_from_normals(N, torch_cuda.as_tensor(g["cf"], device="cuda"), a, b).cpu().numpy()
    assert rel_l2(out, R.field_from_normals(N, g["cf"], a, b)) < 1e-12


def test_generator_draws_have_the_covariance(torch_cuda):
    """Mean |rfft2_ortho(f)|^2 over 64 draws equals C within 4 sigma of the sample mean (interior modes)."""
    from cmblensing_b200.sampling import field_from_covar_single_key
    n, c = 128, 2.5
    gen = torch_cuda.Generator(device="cuda").manual_seed(123)
    cov = torch_cuda.full((n, n // 2 + 1), c, dtype=torch_cuda.float64, device="cuda")
    acc = torch_cuda.zeros_like(cov)
    draws = 64
    for _ in range(draws):
        f = field_from_covar_single_key(n, cov, generator=gen)
        acc += torch_cuda.abs(torch_cuda.fft.rfft2(f, norm="ortho")) ** 2
    interior = (acc / draws)[1:n // 2, 1:n // 2]
    mean = float(interior.mean())
    sigma = c / np.sqrt(interior.numel() * draws)  # |z|^2 of a complex normal: std = mean
    assert abs(mean - c) < 4 * sigma, (mean, c, sigma)


def test_simulate_data_matches_oracle(torch_cuda):
    """d = M B L(phi) f + n on the QU set with given noise normals."""
    from cmblensing_b200.sampling import simulate_data
    g, S = _sets("P", _Mod())
    _, So = _sets("P", R)
    draws = [_normals(10), _normals(11)]
    out = simulate_data(S["field"], S["phi"], S["M"], S["B"], S["Cn"], noise_draws=draws, n=7)
    lensed = R.qu2eb(R.fourier(R.lense_flow(R.map_(R.eb2qu(So["field"])), R.map_(So["phi"]), n=7)))
    noise = [np.fft.rfft2(R.field_from_normals(N, m, *d)) for m, d in zip((g["cn_ee"], g["cn_bb"]), draws)]
    ref = So["M"] * So["B"] * lensed + lensed.replace(polar_matrix_1=noise[0], polar_matrix_2=noise[1])
    for nm in ("polar_matrix_1", "polar_matrix_2"):
        assert rel_l2(getattr(out, nm), getattr(ref, nm)) < 2e-5


@pytest.mark.parametrize("which", ["I", "P"])
def test_mixed_logpdf(torch_cuda, which):
    from cmblensing_b200.mixing import mix
    from cmblensing_b200.statistics import mixed_logpdf
    _, S = _sets(which, _Mod())
    _, So = _sets(which, R)
    D, G = _mixing(which, _Mod())
    Do, Go = _mixing(which, R)
    fmo, pmo = R.mix(So["field"], So["phi"], Do, Go, n=7)
    ref = R.mixed_logpdf(fmo, pmo, So["data"], So["Cn"], So["Cphi"], So["Cf"], So["M"], So["B"], Go, Do, n=7)
    fm, pm = mix(S["field"], S["phi"], D, G, n=7)
    v = mixed_logpdf(fm, pm, S["data"], S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], G, D, n=7)
    assert abs(v - ref) / abs(ref) < 5e-9


def _hmc_inputs(mod):
    g, S = _sets("I", mod)
    D, G = _mixing("I", mod)
    m = load_golden("mix.npz")
    nphi = mod.DiagonalScalar(scalar_matrix=np.ones_like(g["cphi"]) * float(np.median(g["cphi"][1:, 1:])),
                              fourier_weights=S["phi"].fourier_weights)
    return S, D, G, nphi


def test_symplectic_integrate_and_hmc_step(torch_cuda):
    """Two leapfrog steps (T set) from the same momentum: position and delta H match the oracle."""
    from cmblensing_b200.mixing import mix
    from cmblensing_b200.sampling import get_mass_matrix, hmc_step
    S, D, G, nphi = _hmc_inputs(_Mod())
    So, Do, Go, nphio = _hmc_inputs(R)
    mass = get_mass_matrix(S["Cphi"], nphi, G)
    masso = R.get_mass_matrix(So["Cphi"], nphio, Go)
    fmo, pmo = R.mix(So["field"], So["phi"], Do, Go, n=7)
    fm, pm = mix(S["field"], S["phi"], D, G, n=7)
    a, b = _normals(20)
    kw = dict(num_steps=2, step_size=0.01, n=7)
    x_ref, dh_ref, acc_ref = R.hmc_step_from_draws(pmo, False, masso, a, b, 0.0, fmo, So["data"], So["Cn"],
                                                   So["Cphi"], So["Cf"], So["M"], So["B"], Do, Go, **kw)
    x, dh, acc = hmc_step(pm, False, mass, fm, S["data"], S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], D, G,
                          draws=(a, b, 0.0), **kw)
    lp = abs(R.logpdf(So["field"], So["phi"], So["data"], So["Cn"], So["Cphi"], So["Cf"], So["M"], So["B"], n=7))
    assert abs(dh - dh_ref) < 1e-8 * lp, (dh, dh_ref)
    if acc_ref == acc:
        assert rel_l2(x.scalar_matrix, x_ref.scalar_matrix) < 2e-5
    # the proposal itself (independent of the accept decision)
    x2, _, _ = hmc_step(pm, True, mass, fm, S["data"], S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], D, G,
                        draws=(a, b, 0.0), **kw)
    x2_ref, _, _ = R.hmc_step_from_draws(pmo, True, masso, a, b, 0.0, fmo, So["data"], So["Cn"], So["Cphi"],
                                         So["Cf"], So["M"], So["B"], Do, Go, **kw)
    assert rel_l2(x2.scalar_matrix, x2_ref.scalar_matrix) < 2e-5
    assert rel_l2(x2.scalar_matrix, pm.scalar_matrix) > 1e-6  # the step moved


def test_gibbs_sample_f_with_draws(torch_cuda):
    """Constrained realisation (T set, 8 PCG iterations of the reference rule) from the same normals."""
    from cmblensing_b200.sampling import gibbs_sample_f
    _, S = _sets("I", _Mod())
    _, So = _sets("I", R)
    fd, nd = _normals(30), _normals(31)
    ref = R.gibbs_sample_f_from_draws(So["data"] * 0, So["data"], So["phi"], So["Cf"], So["Cn"], So["M"], So["B"],
                                      fd, nd, n=7, maxiter=8)
    out = gibbs_sample_f(S["data"] * 0, S["data"], S["phi"], S["Cf"], S["Cn"], S["M"], S["B"], draws=(fd, nd), n=7,
                         maxiter=8)
    assert rel_l2(out.scalar_matrix, ref.scalar_matrix) < 1e-4
