"""GPU parity of the quadratic-estimate noise (simulate.py:198-385) against the oracle.

Inputs: the reference's golden T and QU operator diagonals (256^2, 2.5'),
with the unlensed spectrum standing in for the lensed one (the reference
takes it from CAMB, which is absent).  The comparison is of the reciprocals,
1/N_phi = sum_ij |d_i d_j rfft2(.)|, as the reference's own test compares
them: at the highest |k| that sum is float64 rounding noise of smooth maps
(1e-16 of its peak), so N_phi there is 1/noise on both sides.  Both sides
are float64 and agree to 1e-10 relative L2.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import lenseflow_ref as R

pytestmark = pytest.mark.gpu
PW = R.pix_width_of(2.5)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _recip(x):
    return np.where(x != 0, 1 / np.where(x != 0, x, 1), 0)


def test_scalar_quadratic_estimate(torch_cuda):
    from cmblensing_b200.quadratic_estimate import scalar_quadratic_estimate
    g = load_golden("infer_I.npz")
    args = (g["cn"], g["cf"], g["cf"], g["m"], g["b"], PW)
    out = scalar_quadratic_estimate(*args).cpu().numpy()
    assert rel_l2(_recip(out), _recip(R.scalar_quadratic_estimate(*args))) < 1e-10


def test_polar_quadratic_estimate(torch_cuda):
    from cmblensing_b200.quadratic_estimate import polar_quadratic_estimate
    g = load_golden("infer_P.npz")
    args = (g["cf_ee"], g["cf_bb"], g["cf_ee"], g["cf_bb"], g["cn_ee"], g["cn_bb"], g["m_ee"], g["m_bb"],
            g["b_ee"], g["b_bb"], PW)
    out = polar_quadratic_estimate(*args).cpu().numpy()
    assert rel_l2(_recip(out), _recip(R.polar_quadratic_estimate(*args))) < 1e-10
