"""The gradient and Wiener-filter workloads on the GPU.

Gradient workload: 256^2 IQU, 3' pixels, d = B L(phi) f + n with a 3' FWHM
beam and white noise of 10 / 14 uK-arcmin (T / QU), no mask, n = 7.  The
FP32 gradients are checked against the float64 oracle's restatement of the
reference (tolerance 2e-5) and against central finite differences of
logpdf (eps = 1e-3 rms) along 16 seeded directions.  For f, logpdf is
quadratic and the gradient uses the exact discrete adjoint: 1e-4.  For phi,
the reference's continuous delta-phi adjoint differs from the exact
derivative by the RK4 discretisation error: 5e-3.  The checkpointed exact
reverse pass (scheme="exact") has no such gap: with the FP64 engine its phi
gradient equals Richardson-extrapolated central differences at the same eps
to 1e-6, and its FP32 gradient matches the oracle's exact restatement to
2e-5.  Directions are seeded Gaussian random fields with the workload's
spectra.

Wiener-filter workload: 512^2 QU, 2' pixels, 1' beam, 2 uK-arcmin noise, a
pixel mask with 30 apodised holes, B-mode prior at 1% of C_EE (the
simulated B is zero); FP32 operator, float64 inner products, true-residual
refinement every 10 iterations.  Stopped at ||r||/||b|| = 1e-8, the
solution must agree with the FP64-engine solution (stopped at 1e-10) to
1e-6.  The 64^2 case compares the GPU PCG with the oracle's float64 PCG.
"""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import lenseflow_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _problem(mod, N, theta, pol, beam_fwhm, noise_t, noise_p, seed=0, nlens=7, mask=None, bb_fraction=0.0):
    """Reference-shaped fields/operators for module ``mod`` (oracle R or cmblensing_b200), data lensed by the oracle."""
    from cmblensing_b200.simulate import inference_problem
    p = inference_problem(N, theta, beam_fwhm=beam_fwhm, noise_t=noise_t, noise_p=noise_p, seed=seed,
                          bb_fraction=bb_fraction)
    pw = R.pix_width_of(theta)
    w = R.get_fourier_weights((N, N))
    kw = dict(nside=N, theta_pix=theta, pix_width=pw, fourier_weights=w)
    ones = np.ones_like(p["beam"])
    if pol == "IP":
        field = mod.FlatS02(scalar_matrix=p["t"], polar_matrix_1=p["e"], polar_matrix_2=p["b"], **kw)
        Z = np.zeros_like(ones)
        blk = lambda tt, ee, bb: mod.BlockTEB(matrix_TT=tt, matrix_TE=Z, matrix_ET=Z, matrix_EE=ee, matrix_BB=bb, **kw)
        Cf = blk(p["cf_tt"], p["cf_ee"], p["cf_bb"])
        Cn = blk(p["cn_t"], p["cn_p"], p["cn_p"])
        B = blk(p["beam"], p["beam"], p["beam"])
        M = blk(ones, ones, ones)
        noise = mod.FlatS02(scalar_matrix=p["n_t"], polar_matrix_1=p["n_e"], polar_matrix_2=p["n_b"], **kw)
    else:
        field = mod.FlatS2(polar_matrix_1=p["e"], polar_matrix_2=p["b"], **kw)
        eb = lambda ee, bb: mod.DiagonalEB(matrix_EE=ee, matrix_BB=bb, **kw)
        Cf = eb(p["cf_ee"], p["cf_bb"])
        Cn = eb(p["cn_p"], p["cn_p"])
        B = eb(p["beam"], p["beam"])
        M = eb(ones, ones)
        noise = mod.FlatS2(polar_matrix_1=p["n_e"], polar_matrix_2=p["n_b"], **kw)
    phi = mod.FlatS0(scalar_matrix=p["phi"], **kw)
    Cphi = mod.DiagonalScalar(scalar_matrix=p["cphi"], **kw)
    # data with the oracle: d = B L f + n (Fourier-diagonal M = 1 here)
    fo = R.FlatS02 if pol == "IP" else R.FlatS2
    f_or = fo(**{k: getattr(field, k) for k in field._matrix_names()}, nside=N, theta_pix=theta, pix_width=pw,
              fourier_weights=w)
    lensed = R.qu2eb(R.fourier(R.lense_flow(R.map_(R.eb2qu(f_or)), R.FlatS0(scalar_matrix=p["phi"], nside=N,
                                                                               theta_pix=theta, pix_width=pw), n=nlens)))
    dmat = {k: p["beam"] * getattr(lensed, k) + getattr(noise, k) for k in field._matrix_names()}
    if mask is not None:  # pixel-space mask on the data
        from cmblensing_b200 import matrix_operators as mo
        M = mo.PixelMask(mask_map=mask, **kw)
        mq = R.map_(R.eb2qu(fo(**dmat, nside=N, theta_pix=theta, pix_width=pw, fourier_weights=w)))
        dm = R.qu2eb(R.fourier(mq.replace(**{k: getattr(mq, k) * mask for k in mq._matrix_names()})))
        dmat = {k: getattr(dm, k) for k in field._matrix_names()}
    data = field.replace(**dmat)
    return dict(field=field, phi=phi, data=data, Cf=Cf, Cn=Cn, B=B, M=M, Cphi=Cphi)


def _as_oracle(S):
    """The same problem as oracle containers."""
    conv = {}
    for k, v in S.items():
        cls = getattr(R, type(v).__name__)
        conv[k] = cls(**{f: getattr(v, f) for f in v._matrix_names()}, nside=v.nside, theta_pix=v.theta_pix,
                      pix_width=v.pix_width, fourier_weights=v.fourier_weights)
    return conv


def _direction(field, seed, kind):
    """A seeded Gaussian-random-field direction with the workload's spectra, in the field's Fourier basis.

    ``kind`` "f": TT for T and EE for E and B; "phi": the phi spectrum.  (Pixel-scale white-noise
    directions in phi are where the reference's continuous delta-phi adjoint is least accurate.)
    """
    from cmblensing_b200.simulate import gaussian_field, gaussian_phi
    N, th = field.nside, field.theta_pix
    mats = {}
    for i, k in enumerate(field._matrix_names()):
        if kind == "phi":
            m = gaussian_phi(N, th, seed=seed)
        else:
            m = gaussian_field(N, th, "TT" if k == "scalar_matrix" else "EE", seed=seed + 97 * i)
        mats[k] = np.fft.rfft2(m / np.sqrt(np.mean(m ** 2)))
    return field.replace(**mats)


def test_gradients_256_IQU(torch_cuda):
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.gradients import grad_phi_logpdf, gradf_logpdf
    from cmblensing_b200.statistics import logpdf

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    S = _problem(Mod, 256, 3.0, "IP", 3.0, 10.0, 14.0, seed=1)
    So = _as_oracle(S)
    f, phi, d = S["field"], S["phi"], S["data"]
    gf = gradf_logpdf(f, phi, d, S["Cf"], S["Cn"], S["M"], S["B"], n=7)
    gf_ref = R.gradf_logpdf(So["field"], So["phi"], So["data"], So["Cf"], So["Cn"], So["M"], So["B"], n=7)
    for k in gf_ref._matrix_names():
        assert rel_l2(getattr(gf, k), getattr(gf_ref, k)) < 2e-5
    gp = grad_phi_logpdf(f, phi, d, S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], n=7)
    gp_ref = R.grad_phi_logpdf(So["field"], So["phi"], So["data"], So["Cn"], So["Cphi"], So["Cf"], So["M"], So["B"],
                               n=7)
    assert rel_l2(gp.scalar_matrix, gp_ref) < 2e-5

    def lp(ff, pp):
        # float64 engine for the finite differences themselves
        from cmblensing_b200 import lense_flow as lfm
        old = lfm.engine.lense_flow_batch
        try:
            lfm.engine.lense_flow_batch = lambda *a, **k: old(*a, **{**k, "precision": "f64"})
            return logpdf(ff, pp, d, S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], n=7)
        finally:
            lfm.engine.lense_flow_batch = old

    rms_f = np.sqrt(np.mean(np.fft.irfft2(f.scalar_matrix, s=(256, 256)) ** 2))
    rms_p = np.sqrt(np.mean(np.fft.irfft2(phi.scalar_matrix, s=(256, 256)) ** 2))
    errs_f, errs_p = [], []
    for k in range(16):
        v = _direction(f, 4000 + k, "f")
        eps = 1e-3 * rms_f
        fd = (lp(f + v * eps, phi) - lp(f - v * eps, phi)) / (2 * eps)
        errs_f.append((fd, R.dot(gf, v)))
        u = _direction(phi, 4100 + k, "phi")
        eps = 1e-3 * rms_p
        fd = (lp(f, phi + u * eps) - lp(f, phi - u * eps)) / (2 * eps)
        errs_p.append((fd, R.dot(gp, u)))
    # errors relative to the typical directional derivative (a direction whose own derivative is
    # small would otherwise dominate a per-direction ratio)
    for pairs, tol in ((errs_f, 1e-4), (errs_p, 5e-3)):
        scale = np.sqrt(np.mean([a * a for a, _ in pairs]))
        worst = max(abs(a - b) for a, b in pairs) / scale
        assert worst < tol, (worst, pairs)


def test_wiener_filter_64_matches_oracle_pcg(torch_cuda):
    """The GPU PCG (FP32 operator, float64 dots) against the oracle's float64 PCG, same stopping rule."""
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.wiener_filter import wiener_filter

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    S = _problem(Mod, 64, 2.0, "P", 1.0, 2.0, 2.0, seed=3, bb_fraction=0.01)
    So = _as_oracle(S)
    x = wiener_filter(S["data"] * 0, S["phi"], S["data"], S["Cf"], S["Cn"], S["M"], S["B"], n=7, rel_tol=1e-8,
                      refine_every=10)
    xo, _ = R.wiener_filter(So["data"] * 0, So["phi"], So["data"], So["Cf"], So["Cn"], So["M"], So["B"], n=7,
                            rel_tol=1e-10)
    for k in xo._matrix_names():
        assert rel_l2(getattr(x, k), getattr(xo, k)) < 1e-6


def test_wiener_filter_512_QU_masked(torch_cuda):
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.simulate import hole_mask
    from cmblensing_b200.wiener_filter import wiener_filter

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    mask = hole_mask(512, 2.0)
    S = _problem(Mod, 512, 2.0, "P", 1.0, 2.0, 2.0, seed=2, mask=mask, bb_fraction=0.01)
    args = (S["data"] * 0, S["phi"], S["data"], S["Cf"], S["Cn"], S["M"], S["B"])
    x32 = wiener_filter(*args, n=7, rel_tol=1e-8, refine_every=10, return_iterations=True, maxiter=1000)
    it32 = wiener_filter.last_iterations
    x64 = wiener_filter(*args, n=7, rel_tol=1e-10, precision="f64", maxiter=2000)
    for k in x64._matrix_names():
        assert rel_l2(getattr(x32, k), getattr(x64, k)) < 1e-6, (k, it32)


@pytest.mark.parametrize("masked", [False, True])
def test_device_wiener_filter_matches_reference_shaped_solver(torch_cuda, masked):
    """The device-resident PCG (precomputed per-mode operators, device scalars) equals the reference-shaped one."""
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.simulate import hole_mask
    from cmblensing_b200.wf_engine import DeviceWienerFilter
    from cmblensing_b200.wiener_filter import wiener_filter

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    S = _problem(Mod, 128, 2.0, "P", 1.0, 2.0, 2.0, seed=5, bb_fraction=0.01,
                 mask=hole_mask(128, 2.0, nholes=5) if masked else None)
    args = (S["data"] * 0, S["phi"], S["data"], S["Cf"], S["Cn"], S["M"], S["B"])
    ref = wiener_filter(*args, n=7, rel_tol=1e-9, refine_every=10)
    wf = DeviceWienerFilter(S["phi"], S["data"], S["Cf"], S["Cn"], S["M"], S["B"], n=7)
    x, it = wf.solve(rel_tol=1e-9, refine_every=10)
    out = wf.to_field(x)
    for k in ref._matrix_names():
        assert rel_l2(getattr(out, k), getattr(ref, k)) < 1e-7, (k, it)
    # and the operator itself against gradf_logpdf(x, d = 0) of the reference-shaped path
    from cmblensing_b200.gradients import gradf_logpdf
    xf = S["data"]
    Ax = wf.apply_A(torch_cuda.stack([torch_cuda.as_tensor(getattr(xf, k), device="cuda")
                                      for k in xf._matrix_names()]))
    g = gradf_logpdf(xf, S["phi"], xf * 0, S["Cf"], S["Cn"], S["M"], S["B"], n=7)
    for i, k in enumerate(g._matrix_names()):  # same kernels; the EB->QU sums round differently before FP32
        assert rel_l2(Ax[i].cpu().numpy(), getattr(g, k)) < 1e-6


def test_batched_wiener_filter_equals_solo_solves(torch_cuda):
    """Three masked problems of one size solved together by the batched CG equal their solo solves."""
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.simulate import hole_mask
    from cmblensing_b200.wf_engine import DeviceWienerFilter

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    probs = []
    for seed in (11, 12, 13):
        S = _problem(Mod, 128, 2.0, "P", 1.0, 2.0, 2.0, seed=seed, bb_fraction=0.01,
                     mask=hole_mask(128, 2.0, nholes=5, seed=seed))
        probs.append(dict(phi=S["phi"], data=S["data"], Cf=S["Cf"], Cn=S["Cn"], M=S["M"], B=S["B"]))
    batch = DeviceWienerFilter(problems=probs, n=7)
    xb, its = batch.solve(rel_tol=1e-9, refine_every=10)
    for i, pr in enumerate(probs):
        solo = DeviceWienerFilter(problems=[pr], n=7)
        xs, _ = solo.solve(rel_tol=1e-9, refine_every=10)
        assert rel_l2(xb[i].cpu().numpy(), xs.cpu().numpy()) < 1e-7, (i, its)


def test_grad_phi_exact_scheme_256_IQU(torch_cuda):
    """grad_phi_logpdf with the checkpointed exact reverse pass: FP64 engine vs Richardson-extrapolated central
    differences (eps = 1e-3 rms and 5e-4 rms, 16 directions) to 1e-6; FP32 engine vs the oracle's exact scheme at
    128^2 to 2e-5."""
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.gradients import grad_phi_logpdf
    from cmblensing_b200.statistics import logpdf

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    S = _problem(Mod, 256, 3.0, "IP", 3.0, 10.0, 14.0, seed=1)
    f, phi, d = S["field"], S["phi"], S["data"]
    args = (d, S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"])
    gp = grad_phi_logpdf(f, phi, *args, n=7, scheme="exact", precision="f64")
    gp_ref = grad_phi_logpdf(f, phi, *args, n=7, scheme="reference", precision="f64")

    def lp(pp):
        from cmblensing_b200 import lense_flow as lfm
        old = lfm.engine.lense_flow_batch
        try:
            lfm.engine.lense_flow_batch = lambda *a, **k: old(*a, **{**k, "precision": "f64"})
            return logpdf(f, pp, d, S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], n=7)
        finally:
            lfm.engine.lense_flow_batch = old

    rms_p = np.sqrt(np.mean(np.fft.irfft2(phi.scalar_matrix, s=(256, 256)) ** 2))
    pairs, pairs_ref = [], []
    for k in range(16):
        u = _direction(phi, 4100 + k, "phi")
        D = lambda e: (lp(phi + u * (e * rms_p)) - lp(phi - u * (e * rms_p))) / (2 * e * rms_p)
        fd = (4 * D(5e-4) - D(1e-3)) / 3
        pairs.append((fd, R.dot(gp, u)))
        pairs_ref.append((fd, R.dot(gp_ref, u)))
    scale = np.sqrt(np.mean([a * a for a, _ in pairs]))
    worst = max(abs(a - b) for a, b in pairs) / scale
    worst_ref = max(abs(a - b) for a, b in pairs_ref) / scale
    assert worst < 1e-6, (worst, worst_ref)
    assert worst_ref > 10 * worst  # the reference scheme's RK4 gap is visible at this precision

    S = _problem(Mod, 128, 3.0, "IP", 3.0, 10.0, 14.0, seed=2)
    So = _as_oracle(S)
    g32 = grad_phi_logpdf(S["field"], S["phi"], S["data"], S["Cn"], S["Cphi"], S["Cf"], S["M"], S["B"], n=7,
                          scheme="exact")
    go = R.grad_phi_logpdf(So["field"], So["phi"], So["data"], So["Cn"], So["Cphi"], So["Cf"], So["M"], So["B"], n=7,
                           scheme="exact")
    assert rel_l2(g32.scalar_matrix, go) < 2e-5


@pytest.mark.parametrize("C,batched", [(1, False), (2, True), (3, True), (3, False)])
def test_modes_apply_matches_torch(torch_cuda, C, batched):
    """lf_modes_apply (the Wiener filter's fused per-mode operator product) against torch, zero blocks skipped,
    in place and with the Y term."""
    import ctypes
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    from cmblensing_b200.wf_engine import _nonzero_mask
    lib = nat.load()
    B, N = 3, 64
    H = N // 2 + 1
    g = torch.Generator(device="cpu").manual_seed(C)
    W = torch.randn(((B,) if batched else ()) + (C, C, N, H), generator=g, dtype=torch.float64)
    if C == 3:
        W[..., 0, 2, :, :] = 0
        W[..., 2, 0, :, :] = 0
    W = W.cuda()
    X = torch.randn((B, C, N, H), generator=g, dtype=torch.complex128).cuda()
    Y = torch.randn((B, C, N, H), generator=g, dtype=torch.complex128).cuda()
    Wb = W if batched else W.unsqueeze(0).expand(B, *W.shape)
    ref = 0.5 * torch.einsum("bijnh,bjnh->binh", Wb.to(torch.complex128), X) - 2.0 * Y
    nz = _nonzero_mask(W)
    if C == 3:
        assert not nz & (1 << 2) and not nz & (1 << 6)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.empty_like(X)
    assert lib.lf_modes_apply(vp(W), int(batched), nz, vp(X), vp(Y), vp(out), B, C, N * H, 0.5, -2.0, st) == 0
    Xi = X.clone()  # in place: out aliases X
    assert lib.lf_modes_apply(vp(W), int(batched), nz, vp(Xi), vp(Y), vp(Xi), B, C, N * H, 0.5, -2.0, st) == 0
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < 1e-14
    assert torch.equal(out, Xi)


def test_wiener_filter_graph_replay_equals_eager(torch_cuda):
    """The CG blocks replayed from a captured CUDA graph give the eager iterations' iterates and counts."""
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.simulate import hole_mask
    from cmblensing_b200.wf_engine import DeviceWienerFilter

    class Mod:
        FlatS0, FlatS2, FlatS02 = cl.FlatS0, cl.FlatS2, cl.FlatS02
        DiagonalScalar, DiagonalEB, BlockTEB = mo.DiagonalScalar, mo.DiagonalEB, mo.BlockTEB

    probs = []
    for seed in (21, 22):
        S = _problem(Mod, 128, 2.0, "P", 1.0, 2.0, 2.0, seed=seed, bb_fraction=0.01,
                     mask=hole_mask(128, 2.0, nholes=5, seed=seed))
        probs.append(dict(phi=S["phi"], data=S["data"], Cf=S["Cf"], Cn=S["Cn"], M=S["M"], B=S["B"]))
    wf = DeviceWienerFilter(problems=probs, n=7)
    xg, itg = wf.solve(rel_tol=1e-8, refine_every=10, use_graphs=True)
    assert wf.graph_blocks >= 1
    xe, ite = wf.solve(rel_tol=1e-8, refine_every=10, use_graphs=False)
    assert wf.graph_blocks == 0
    assert itg == ite
    assert torch_cuda.equal(xg, xe)
