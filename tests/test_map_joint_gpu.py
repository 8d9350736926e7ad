"""GPU parity of the MAP-joint loop (cmb_lensing/map_joint.py:19-98) against the oracle.

The golden T set (256^2, 2.5', DC/Nyquist weight 1) with the reference's
mixing diagonal D and quadratic-estimate noise Nphi; n = 7 RK4 steps and 8
iterations of the reference-rule Wiener filter per step, so the oracle runs
in seconds.  Tolerances: -logpdf values to 5e-9 relative (FP32 lensing, as
the logpdf tests); the loop's f to 1e-4 (the Wiener-filter tests' bound
after a truncated PCG) and phi to 1e-2 (the phi step amplifies f's relative
error about 50-fold, measured on the oracle).  The batched line search is checked against
the reference's BFGS step: same alpha to 10%, -logpdf no worse than BFGS's
beyond FP32 rounding.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import lenseflow_ref as R
from test_inference_gpu import _Mod, _sets
from test_mixing_gpu import _mixing

pytestmark = pytest.mark.gpu
KW = dict(n=7, wf_maxiter=8)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _problem(mod):
    g, S = _sets("I", mod)
    D, _ = _mixing("I", mod)
    qe = mod.DiagonalScalar(scalar_matrix=load_golden("mix.npz")["nphi_t"], fourier_weights=S["phi"].fourier_weights)
    return S, D, qe


def test_neg_logpdf_along_matches_oracle(torch_cuda):
    from cmblensing_b200.map_joint import get_scalar_identity, neg_logpdf_along, phi_gradient_hessian
    from cmblensing_b200.matrix_operators import pinv
    from cmblensing_b200.mixing import mix
    S, D, qe = _problem(_Mod())
    So, Do, qeo = _problem(R)
    G, Go = get_scalar_identity(D), R.get_scalar_identity(Do)
    H, Ho = pinv(phi_gradient_hessian(S["Cphi"], qe)), R.pinv(R.phi_gradient_hessian(So["Cphi"], qeo))
    fmo, pmo = R.mix(So["field"], So["phi"], Do, Go, n=7)
    fm, pm = mix(S["field"], S["phi"], D, G, n=7)
    # a search direction whose preconditioned step is ~5% of phi
    go = pmo.replace(scalar_matrix=0.05 * (R.pinv(So["Cphi"]) * pmo).scalar_matrix)
    gd = pm.replace(scalar_matrix=go.scalar_matrix)
    alphas = [0.0, 0.5, 1.0, 2.0]
    out = neg_logpdf_along(alphas, gd, fm, pm, S["data"], S["B"], S["M"], S["Cf"], S["Cphi"], S["Cn"], D, G, H, n=7)
    for a, v in zip(alphas, out):
        ref = R.logpdf_at_phi_new(a, go, fmo, pmo, So["data"], So["B"], So["M"], So["Cf"], So["Cphi"], So["Cn"], Do,
                                  Go, Ho, n=7)
        assert abs(v - ref) / abs(ref) < 5e-9, (a, v, ref)


def test_map_joint_constant_step_matches_oracle(torch_cuda):
    from cmblensing_b200.map_joint import DataSet, map_joint
    S, D, qe = _problem(_Mod())
    So, Do, qeo = _problem(R)
    ds = DataSet(data=S["data"], noise_covariance=S["Cn"], mixing_d=D, field_covariance=S["Cf"],
                 phi_covariance=S["Cphi"], quadratic_estimate=qe, mask=S["M"], beam=S["B"])
    f, phi = map_joint(ds, num_steps=2, constant_step=True, **KW)
    fo, phio = R.map_joint(So["data"], So["Cn"], Do, So["Cf"], So["Cphi"], qeo, So["M"], So["B"], num_steps=2,
                           constant_step=True, **KW)
    assert rel_l2(f.scalar_matrix, fo.scalar_matrix) < 1e-4
    # the phi step subtracts a prior term from a data term of similar size: on the oracle, a 1e-4 relative
    # perturbation of f moves the step by 4.9e-3, so f's FP32 differences above show up ~50x larger in phi
    assert rel_l2(phi.scalar_matrix, phio.scalar_matrix) < 1e-2


def test_batched_line_search_against_bfgs(torch_cuda):
    """One MAP step: the batched search's alpha and -logpdf against the reference's scipy BFGS on the oracle."""
    from scipy.optimize import minimize
    from cmblensing_b200.map_joint import DataSet, map_joint
    S, D, qe = _problem(_Mod())
    So, Do, qeo = _problem(R)
    ds = DataSet(data=S["data"], noise_covariance=S["Cn"], mixing_d=D, field_covariance=S["Cf"],
                 phi_covariance=S["Cphi"], quadratic_estimate=qe, mask=S["M"], beam=S["B"])
    hist = []
    map_joint(ds, num_steps=1, history=hist, **KW)
    alpha_d, value_d = hist[0]
    # the oracle's first step, with the reference's BFGS line search
    Go = R.get_scalar_identity(Do)
    Ho = R.pinv(R.phi_gradient_hessian(So["Cphi"], qeo))
    f, _ = R.wiener_filter(So["data"] * 0, R.zero_scalar_field_like(So["data"]), So["data"], So["Cf"], So["Cn"],
                           So["M"], So["B"], n=7, maxiter=8)
    fm, pm = R.mix(f, R.zero_scalar_field_like(So["data"]), Do, Go, n=7)
    g = pm.replace(scalar_matrix=R.mixed_grad_phi_logpdf(fm, pm, So["data"], So["Cn"], So["Cphi"], So["Cf"],
                                                         So["M"], So["B"], Do, Go, n=7))
    obj = lambda a: R.logpdf_at_phi_new(float(np.ravel(a)[0]), g, fm, pm, So["data"], So["B"], So["M"], So["Cf"],
                                        So["Cphi"], So["Cn"], Do, Go, Ho, n=7)
    res = minimize(obj, 1.0, method="BFGS")
    alpha_o, value_o = float(res.x[0]), float(res.fun)
    assert abs(alpha_d - alpha_o) < 0.1 * abs(alpha_o), (alpha_d, alpha_o)
    assert value_d <= value_o + 1e-8 * abs(value_o), (value_d, value_o)
