"""GPU parity of the CUDA LenseFlow path against the float64 oracle.

Tolerance (from the workload spec): relative L2 error <= 1e-5 for the FP32
engine; <= 1e-10 for the FP64 engine.  Inputs are seeded Gaussian random
fields with the workloads' spectra (cmblensing_b200.simulate).
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import lenseflow_ref as R

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL64 = 1e-10


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _inputs(N, theta, C, B=1, seed0=0):
    from cmblensing_b200.simulate import lens_batch
    return lens_batch(N, theta, B, C, seed0=seed0)


def _oracle(f, phi, pw, n, direction, adjoint):
    derivs = R.phi_derivatives(phi, pw)
    return np.stack([R.primal_lense_flow(f[c], phi, pw, n, direction, adjoint, derivs) for c in range(f.shape[0])])


def _engine(torch, f, phis, pw, n, direction, adjoint, precision="f32"):
    from cmblensing_b200 import engine
    ft = torch.as_tensor(f, device="cuda")
    pt = torch.as_tensor(phis, device="cuda")
    return engine.lense_flow_batch(ft, pt, pw, n=n, direction=direction, adjoint=adjoint,
                                   precision=precision).double().cpu().numpy()


@pytest.mark.parametrize("N,theta,C", [(64, 3.0, 1), (128, 3.0, 1), (128, 3.0, 2), (64, 3.0, 3), (256, 3.0, 2),
                                       (512, 2.0, 2)])
@pytest.mark.parametrize("direction,adjoint", [(1, False), (-1, False), (1, True), (-1, True)])
def test_lens_matches_oracle(torch_cuda, N, theta, C, direction, adjoint):
    f, phis = _inputs(N, theta, C)
    pw = R.pix_width_of(theta)
    got = _engine(torch_cuda, f, phis, pw, 7, direction, adjoint)[0]
    ref = _oracle(f[0], phis[0], pw, 7, direction, adjoint)
    for c in range(C):
        assert rel_l2(got[c], ref[c]) < TOL32, (c, rel_l2(got[c], ref[c]))


@pytest.mark.parametrize("C,direction,adjoint", [(2, 1, False), (2, -1, False), (1, 1, True), (3, -1, True)])
def test_p_plane_and_derivative_plane_paths(torch_cuda, C, direction, adjoint):
    """A workspace of lf_workspace_bytes_n selects the stage-time p planes; one of lf_workspace_bytes the
    five-plane path.  Both match the oracle and each other (the p planes are formed in float64)."""
    import torch
    from cmblensing_b200 import engine
    N, theta, n = 128, 3.0, 7
    f, phis = _inputs(N, theta, C, B=2, seed0=5)
    pw = R.pix_width_of(theta)
    plan = engine.get_plan(N, C, pw)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    small = plan.workspace_bytes(2, adjoint)
    full = plan.workspace_bytes(2, adjoint, n)
    assert full > small
    outs = []
    for nbytes in (small, full):
        ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        outs.append(plan.lense_flow(ft, planes, n=n, direction=direction, adjoint=adjoint,
                                    workspace=ws).double().cpu().numpy())
    for b in range(2):
        ref = _oracle(f[b], phis[b], pw, n, direction, adjoint)
        for out in outs:
            for c in range(C):
                assert rel_l2(out[b, c], ref[c]) < TOL32
    assert rel_l2(outs[0], outs[1]) < 1e-6


def test_qu512_stage_waits_complete(torch_cuda):
    """The 512^2 QU stage kernels (standard and adjoint) stage their operands with bulk copies; every block's
    bounded wait completes."""
    import torch
    from cmblensing_b200 import engine
    engine.wait_timeouts(reset=True)
    f, phis = _inputs(512, 2.0, 2, B=3, seed0=9)
    pw = R.pix_width_of(2.0)
    for direction in (1, -1):
        for adjoint in (False, True):
            _engine(torch, f, phis, pw, 7, direction, adjoint)
    torch.cuda.synchronize()
    assert engine.wait_timeouts() == 0


def test_lens_1024_T(torch_cuda):
    f, phis = _inputs(1024, 2.0, 1)
    pw = R.pix_width_of(2.0)
    got = _engine(torch_cuda, f, phis, pw, 7, 1, False)[0]
    ref = _oracle(f[0], phis[0], pw, 7, 1, False)
    assert rel_l2(got[0], ref[0]) < TOL32


@pytest.mark.parametrize("adjoint", [False, True])
def test_lens_fp64_engine(torch_cuda, adjoint):
    f, phis = _inputs(128, 3.0, 2)
    pw = R.pix_width_of(3.0)
    got = _engine(torch_cuda, f, phis, pw, 7, 1, adjoint, precision="f64")[0]
    ref = _oracle(f[0], phis[0], pw, 7, 1, adjoint)
    for c in range(2):
        assert rel_l2(got[c], ref[c]) < TOL64


def test_phi_fourier_basis(torch_cuda):
    """phi given as an rfft2 matrix (lense_flow.py:299-300) gives the same lens."""
    f, phis = _inputs(128, 3.0, 1)
    pw = R.pix_width_of(3.0)
    phif = np.fft.rfft2(phis[0])[None]
    got = _engine(torch_cuda, f, phif, pw, 7, 1, False)[0]
    ref = _oracle(f[0], phif[0], pw, 7, 1, False)
    assert rel_l2(got[0], ref[0]) < TOL32


def test_phi_fourier_non_hermitian_columns(torch_cuda):
    """A Fourier phi with arbitrary imaginary parts on its DC/Nyquist columns: irfft2 semantics."""
    f, phis = _inputs(64, 3.0, 1)
    pw = R.pix_width_of(3.0)
    rng = np.random.default_rng(5)
    phif = np.fft.rfft2(phis[0])
    phif[:, 0] += 1j * rng.standard_normal(64) * np.abs(phif[:, 0]).mean() * 0.005
    phif[:, -1] += 1j * rng.standard_normal(64) * np.abs(phif[:, 1]).mean() * 0.005
    got = _engine(torch_cuda, f, phif[None], pw, 7, 1, False)[0]
    ref = _oracle(f[0], phif, pw, 7, 1, False)
    assert rel_l2(got[0], ref[0]) < TOL32


def test_golden_forward_T_256(torch_cuda):
    """The engine against the reference's Julia golden (256^2, 2.5', n=7)."""
    g = load_golden("lens_I.npz")
    pw = R.pix_width_of(float(g["theta_pix"]))
    t = np.fft.irfft2(g["t"], s=(256, 256))
    phi = np.fft.irfft2(g["phi"], s=(256, 256))
    got = _engine(torch_cuda, t[None, None], phi[None], pw, 7, 1, False)[0, 0]
    r, c = g["idx"]
    assert rel_l2(np.fft.rfft2(got)[r, c], g["t_lensed"]) < TOL32


def test_golden_forward_QU_256(torch_cuda):
    g = load_golden("lens_P.npz")
    pw = R.pix_width_of(float(g["theta_pix"]))
    qu = R.map_(R.eb2qu(R.FlatS2(polar_matrix_1=g["e"], polar_matrix_2=g["b"])))
    phi = np.fft.irfft2(g["phi"], s=(256, 256))
    f = np.stack([qu.polar_matrix_1, qu.polar_matrix_2])[None]
    got = _engine(torch_cuda, f, phi[None], pw, 7, 1, False)[0]
    out = R.qu2eb(R.fourier(R.FlatS2(polar_matrix_1=got[0], polar_matrix_2=got[1], basis=R.Basis.MAP)))
    r, c = g["idx"]
    assert rel_l2(out.polar_matrix_1[r, c], g["e_lensed"]) < TOL32
    assert rel_l2(out.polar_matrix_2[r, c], g["b_lensed"]) < TOL32


def test_batch_equals_single(torch_cuda):
    """Each map of a batch equals the same map lensed alone (bit-exact: same kernels, same tiles)."""
    f, phis = _inputs(128, 3.0, 2, B=5)
    pw = R.pix_width_of(3.0)
    batch = _engine(torch_cuda, f, phis, pw, 7, 1, False)
    for i in (0, 3):
        one = _engine(torch_cuda, f[i:i + 1], phis[i:i + 1], pw, 7, 1, False)
        assert np.array_equal(one[0], batch[i])


@pytest.mark.parametrize("direction,adjoint", [(1, False), (-1, False), (1, True)])
def test_qu512_batch_maps_equal_solo_and_oracle(torch_cuda, direction, adjoint):
    """The bench's shape (512^2 QU, p planes, the paired row kernels) at B = 4 distinct maps: every map of the
    batch is bit-identical to the same map lensed alone (the batch index of k_row_pair / k_row_pair_adj and of
    k_p_planes), and the last map matches the float64 oracle."""
    import torch
    from cmblensing_b200 import engine
    N, theta, C, B, n = 512, 2.0, 2, 4, 7
    f, phis = _inputs(N, theta, C, B=B, seed0=40)
    pw = R.pix_width_of(theta)
    plan = engine.get_plan(N, C, pw)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    ws = torch.empty(plan.workspace_bytes(B, adjoint, n), dtype=torch.uint8, device="cuda")  # the p-plane path
    batch = plan.lense_flow(ft, planes, n=n, direction=direction, adjoint=adjoint, workspace=ws)
    for i in range(B):
        one = plan.lense_flow(ft[i:i + 1], planes[i:i + 1], n=n, direction=direction, adjoint=adjoint)
        assert torch.equal(one[0], batch[i]), i
    ref = _oracle(f[B - 1], phis[B - 1], pw, n, direction, adjoint)
    got = batch[B - 1].double().cpu().numpy()
    for c in range(C):
        assert rel_l2(got[c], ref[c]) < TOL32, (c, rel_l2(got[c], ref[c]))


def test_lense_flow_backwards_qu_map_phi_matches_oracle(torch_cuda):
    """The reference-shaped reverse pass on a QU field with a MAP phi and a MAP cotangent: the returned delta-f
    has Q and U swapped as the reference's output_like_input writes them (lense_flow.py:143-152), and both
    outputs go through the MAP branch of undo_inner_product (fields.py:147-154) -- against the oracle's
    lense_flow_backwards.  The reference's default Fourier weights (0.5 on the DC/Nyquist columns) are used."""
    import cmblensing_b200 as cl
    from cmblensing_b200.lense_flow import lense_flow_backwards
    N, theta, n = 128, 3.0, 7
    f, phis = _inputs(N, theta, 2, seed0=12)
    pw = R.pix_width_of(theta)
    rng = np.random.default_rng(13)
    cot = rng.standard_normal((2, N, N))
    lensed = _oracle(f[0], phis[0], pw, n, 1, False)
    kw = dict(nside=N, theta_pix=theta, pix_width=pw)
    mk = lambda mod, a: mod.FlatS2(polar_matrix_1=a[0], polar_matrix_2=a[1], basis=mod.Basis.MAP, **kw)
    phi_e = cl.FlatS0(scalar_matrix=phis[0], basis=cl.Basis.MAP, **kw)
    phi_o = R.FlatS0(scalar_matrix=phis[0], basis=R.Basis.MAP, **kw)
    df, dphi = lense_flow_backwards(mk(cl, lensed), phi_e, mk(cl, cot), n=n, direction=1)
    df_o, dphi_o = R.lense_flow_backwards(mk(R, lensed), phi_o, mk(R, cot), n=n, direction=1)
    assert isinstance(df.polar_matrix_1, np.ndarray) and df.polar_matrix_1.shape == (N, N)
    # the swap: polar_matrix_1 holds the U component's delta (compare with the unswapped engine output)
    df_plain, _ = lense_flow_backwards(mk(cl, lensed), phi_e, mk(cl, cot), n=n, direction=1, swap_qu=False)
    assert np.array_equal(df.polar_matrix_1, df_plain.polar_matrix_2)
    assert np.array_equal(df.polar_matrix_2, df_plain.polar_matrix_1)
    assert rel_l2(df.polar_matrix_1, df_o.polar_matrix_1) < 1e-5
    assert rel_l2(df.polar_matrix_2, df_o.polar_matrix_2) < 1e-5
    assert dphi.scalar_matrix.shape == (N, N)
    assert rel_l2(dphi.scalar_matrix, dphi_o.scalar_matrix) < 2e-5


def test_round_trip_512_QU(torch_cuda):
    """Full-size property: ||L^-1 L f - f|| / ||f|| equals the float64 oracle's own RK4 round-trip residual."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(512, 2.0, 2, B=2)
    pw = R.pix_width_of(2.0)
    plan = engine.get_plan(512, 2, pw)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    lensed = plan.lense_flow(ft, planes, n=7)
    back = plan.lense_flow(lensed, planes, n=7, direction=-1)
    err = float((back - ft).norm() / ft.norm())
    num = den = 0.0
    for b in range(2):
        L = _oracle(f[b], phis[b], pw, 7, 1, False)
        back_ref = _oracle(L, phis[b], pw, 7, -1, False)
        num += float(np.sum((back_ref - f[b]) ** 2))
        den += float(np.sum(f[b] ** 2))
    ref = np.sqrt(num / den)
    assert abs(err - ref) / ref < 1e-2, (err, ref)


def test_qu512_paired_adjoint(torch_cuda):
    """The 512^2 QU adjoint with p planes (one paired transform for both rates) matches the five-plane adjoint,
    and <L a, L a> == <a, L^T L a> to FP32 rounding."""
    import torch
    from cmblensing_b200 import engine
    N, theta, n, B = 512, 2.0, 7, 2
    f, phis = _inputs(N, theta, 2, B=B, seed0=21)
    pw = R.pix_width_of(theta)
    plan = engine.get_plan(N, 2, pw)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    a = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    rng = np.random.default_rng(4)
    b = torch.as_tensor(rng.standard_normal(f.shape), device="cuda", dtype=torch.float32)
    outs = []
    for nbytes in (plan.workspace_bytes(B, True), plan.workspace_bytes(B, True, n)):
        ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        outs.append(plan.lense_flow(b, planes, n=n, adjoint=True, workspace=ws).double())
    assert float(torch.linalg.vector_norm(outs[0] - outs[1]) / torch.linalg.vector_norm(outs[0])) < 1e-6
    # <L a, L a> == <a, L^T (L a)>: positive on both sides, so FP32 rounding is not amplified by cancellation
    La = plan.lense_flow(a, planes, n=n)
    LTLa = plan.lense_flow(La, planes, n=n, adjoint=True).double()
    for m in range(B):
        lhs = float((La[m].double() ** 2).sum())
        rhs = float((a[m].double() * LTLa[m]).sum())
        assert abs(lhs - rhs) / abs(lhs) < 1e-5, (m, lhs, rhs)


def test_adjoint_dot_product(torch_cuda):
    """<L a, b> == <a, L^T b> for the discrete operator (the adjoint RHS is the exact transpose)."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(128, 3.0, 1, B=1)
    pw = R.pix_width_of(3.0)
    rng = np.random.default_rng(3)
    a = torch.as_tensor(f, device="cuda", dtype=torch.float64)
    b = torch.as_tensor(rng.standard_normal(f.shape), device="cuda", dtype=torch.float64)
    plan = engine.get_plan(128, 1, pw, "f64")
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    La = plan.lense_flow(a, planes, n=7)
    LTb = plan.lense_flow(b, planes, n=7, adjoint=True)
    lhs = float((La * b).sum())
    rhs = float((a * LTb).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-10


def test_in_place_and_f64_io(torch_cuda):
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(64, 3.0, 2, B=2)
    pw = R.pix_width_of(3.0)
    plan = engine.get_plan(64, 2, pw)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    x64 = torch.as_tensor(f, device="cuda")
    ref = plan.lense_flow(x64, planes, n=7)  # float64 in and out, FP32 compute
    assert ref.dtype == torch.float64
    x = x64.clone()
    plan.lense_flow(x, planes, n=7, out=x)
    assert torch.equal(x, ref)


def test_zero_steps_identity_and_empty_batch(torch_cuda):
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(64, 3.0, 1, B=1)
    pw = R.pix_width_of(3.0)
    plan = engine.get_plan(64, 1, pw)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    x = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    assert torch.equal(plan.lense_flow(x, planes, n=0), x)
    empty = torch.empty((0, 1, 64, 64), device="cuda")
    assert plan.lense_flow(empty, planes[:0], n=7).shape == (0, 1, 64, 64)


def test_singular_phi_is_reported(torch_cuda):
    import torch
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import gaussian_phi
    phi = gaussian_phi(128, 3.0, seed=7, deflection_arcmin=2.5, spectrum="literal")
    plan = engine.get_plan(128, 1, R.pix_width_of(3.0))
    with pytest.raises(nat.SingularMagnificationError):
        plan.phi_planes(torch.as_tensor(phi[None], device="cuda"))


def test_min_det_matches_host(torch_cuda):
    import torch
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import gaussian_phi, min_magnification_det
    phi = gaussian_phi(256, 3.0, seed=11)
    plan = engine.get_plan(256, 1, R.pix_width_of(3.0))
    plan.phi_planes(torch.as_tensor(phi[None], device="cuda"))
    assert abs(plan.last_min_det[0] - min_magnification_det(phi, 3.0)) < 1e-5


def test_bad_shapes_raise(torch_cuda):
    import torch
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    plan = engine.get_plan(64, 1, R.pix_width_of(3.0))
    with pytest.raises(nat.LenseFlowError):
        plan.phi_planes(torch.zeros((1, 64, 40), device="cuda", dtype=torch.float64))
    planes = torch.zeros((1, 5, 64, 64), device="cuda")
    with pytest.raises(nat.LenseFlowError):
        plan.lense_flow(torch.zeros((1, 2, 64, 64), device="cuda"), planes)


def test_reference_shaped_api(torch_cuda):
    """lense_flow(field, phi, n, direction, adjoint) on reference-shaped containers."""
    import cmblensing_b200 as cl
    from cmblensing_b200.lense_flow import lense_flow
    f, phis = _inputs(128, 3.0, 2)
    pw = R.pix_width_of(3.0)
    field = cl.FlatS2(nside=128, theta_pix=3.0, pix_width=pw, basis=cl.Basis.MAP,
                      polar_matrix_1=f[0, 0], polar_matrix_2=f[0, 1])
    phi = cl.FlatS0(nside=128, theta_pix=3.0, pix_width=pw, basis=cl.Basis.MAP, scalar_matrix=phis[0])
    out = lense_flow(field, phi, n=7, direction=cl.INVERSE_LENSE)
    assert isinstance(out, cl.FlatS2) and isinstance(out.polar_matrix_1, np.ndarray)
    ref = _oracle(f[0], phis[0], pw, 7, -1, False)
    assert rel_l2(out.polar_matrix_1, ref[0]) < TOL32
    assert rel_l2(out.polar_matrix_2, ref[1]) < TOL32


@pytest.mark.parametrize("B,chunks,sizes", [(5, 2, None), (8, 4, None), (8, 4, [1, 2, 4, 1])])
def test_host_pipeline_matches_device_call(torch_cuda, B, chunks, sizes):
    """The pipelined host-buffer path (three streams, double-buffered chunks) equals the device call per map."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(128, 3.0, 2, B=B)
    pw = R.pix_width_of(3.0)
    plan = engine.get_plan(128, 2, pw)
    pipe = engine.HostPipeline(plan, B, chunks=chunks, chunk_sizes=sizes)
    fh = torch.from_numpy(f).pin_memory()
    ph = torch.from_numpy(phis).pin_memory()
    oh = torch.empty_like(fh).pin_memory()
    for _ in range(3):  # eager, graph capture, graph replay; every slot reused
        oh.zero_()
        pipe(fh, ph, oh, n=7)
        torch.cuda.synchronize()
    # float32 plans: the pipeline forms the p planes in the phi precompute (phi_pp + lense_flow_pp)
    ref = plan.lense_flow_pp(torch.as_tensor(f, device="cuda"), plan.phi_pp(torch.as_tensor(phis, device="cuda"), 7),
                             7)
    assert torch.equal(oh, ref.cpu())


def test_host_pipeline_overlapped_calls(torch_cuda):
    """wait=False calls queue behind each other (slot reuse ordered by events); each output equals the device
    call, and wait() joins them."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(128, 3.0, 2, B=6, seed0=11)
    pw = R.pix_width_of(3.0)
    plan = engine.get_plan(128, 2, pw)
    pipe = engine.HostPipeline(plan, 3, chunks=3, slots=2)
    halves = [(torch.from_numpy(f[k * 3:(k + 1) * 3].copy()).pin_memory(),
               torch.from_numpy(phis[k * 3:(k + 1) * 3].copy()).pin_memory()) for k in range(2)]
    outs = [torch.empty((3, 2, 128, 128), dtype=torch.float64).pin_memory() for _ in range(2)]
    for rep in range(4):  # eager, capture, replay; the two rings alternate
        for o in outs:
            o.zero_()
        for k in range(2):
            pipe(halves[k][0], halves[k][1], outs[k], n=7, wait=False)
        pipe.wait()
        torch.cuda.synchronize()
        for k in range(2):
            ref = plan.lense_flow_pp(torch.as_tensor(f[k * 3:(k + 1) * 3], device="cuda"),
                                     plan.phi_pp(torch.as_tensor(phis[k * 3:(k + 1) * 3], device="cuda"), 7), 7)
            assert torch.equal(outs[k], ref.cpu()), (rep, k)


def test_host_pipeline_reports_singular_phi(torch_cuda):
    import torch
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import gaussian_phi
    f, phis = _inputs(128, 3.0, 1, B=3)
    phis[1] = gaussian_phi(128, 3.0, seed=7, spectrum="literal")
    plan = engine.get_plan(128, 1, R.pix_width_of(3.0))
    pipe = engine.HostPipeline(plan, 3, chunks=3)
    with pytest.raises(nat.SingularMagnificationError):
        pipe(torch.from_numpy(f).pin_memory(), torch.from_numpy(phis).pin_memory(),
             torch.empty(f.shape, dtype=torch.float64).pin_memory(), n=7)
    # queued without waiting, the error surfaces at wait()
    pipe(torch.from_numpy(f).pin_memory(), torch.from_numpy(phis).pin_memory(),
         torch.empty(f.shape, dtype=torch.float64).pin_memory(), n=7, wait=False)
    with pytest.raises(nat.SingularMagnificationError):
        pipe.wait()


# ------------------------------------------- p planes formed in the phi precompute
@pytest.mark.parametrize("N,theta,C", [(64, 3.0, 1), (128, 3.0, 2), (256, 3.0, 3), (512, 2.0, 2), (1024, 2.0, 1)])
def test_phi_pp_lens_matches_oracle_and_p_plane_path(torch_cuda, N, theta, C):
    """lf_phi_precompute_pp + lf_lense_flow_pp: one ascending set of p planes serves the forward, inverse and
    adjoint lens; every result matches the oracle (1e-5) and the lf_lense_flow p-plane path (1e-6: the p planes
    differ only in rounding: float32 arithmetic on float64 derivatives there, float64 arithmetic on float32
    planes here); the optional derivative planes
    equal lf_phi_precompute's bit for bit, and the magnification minimum agrees.  Without the derivative planes
    (float32 spectra between the transforms) the p planes agree to 1e-6 and serve the same lenses."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(N, theta, C, B=2, seed0=50)
    pw = R.pix_width_of(theta)
    plan = engine.get_plan(N, C, pw)
    ph = torch.as_tensor(phis, device="cuda")
    planes = plan.phi_planes(ph)
    md_planes = list(plan.last_min_det)
    planes_pp = torch.empty_like(planes)
    pp = plan.phi_pp(ph, 7, planes_out=planes_pp)
    assert torch.equal(planes_pp, planes)
    for a, b in zip(plan.last_min_det, md_planes):
        assert abs(a - b) < 1e-6 * max(1.0, abs(b))
    # without the derivative planes the spectra between the column and row transforms are float32: the p planes
    # move by float32 rounding only, and the magnification minimum with them
    pp32 = plan.phi_pp(ph, 7)
    assert float((pp32 - pp).norm() / pp.norm()) < 1e-6
    for a, b in zip(plan.last_min_det, md_planes):
        assert abs(a - b) < 1e-5 * max(1.0, abs(b))
    ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    cases = [(1, False), (-1, False), (1, True)] if N <= 512 else [(1, False)]
    for direction, adjoint in cases:
        ref_pp = plan.lense_flow(ft, planes, n=7, direction=direction, adjoint=adjoint)
        ref = _oracle(f[1], phis[1], pw, 7, direction, adjoint)
        for p_set in (pp, pp32):
            got = plan.lense_flow_pp(ft, p_set, 7, direction=direction, adjoint=adjoint)
            assert float((got - ref_pp).norm() / ref_pp.norm()) < 1e-6
            g = got[1].double().cpu().numpy()
            for c in range(C):
                assert rel_l2(g[c], ref[c]) < TOL32, (direction, adjoint, c)


def test_phi_pp_reports_singular_phi_and_rejects_f64_plans(torch_cuda):
    import torch
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import gaussian_phi
    phi = gaussian_phi(128, 3.0, seed=7, deflection_arcmin=2.5, spectrum="literal")
    plan = engine.get_plan(128, 1, R.pix_width_of(3.0))
    with pytest.raises(nat.SingularMagnificationError):
        plan.phi_pp(torch.as_tensor(phi[None], device="cuda"), 7)
    plan64 = engine.get_plan(128, 1, R.pix_width_of(3.0), "f64")
    with pytest.raises(nat.LenseFlowError) as e:
        plan64.phi_pp(torch.as_tensor(phi[None], device="cuda"), 7, check_det=False)
    assert e.value.status == nat.LF_ERR_BAD_DTYPE


def test_phi_pp_fourier_basis_equals_map_basis(torch_cuda):
    """A Fourier phi (the rfft2 of a real map) and the map itself give the same p planes and lens."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(128, 3.0, 2, B=2, seed0=60)
    plan = engine.get_plan(128, 2, R.pix_width_of(3.0))
    pp_map = plan.phi_pp(torch.as_tensor(phis, device="cuda"), 7)
    pp_four = plan.phi_pp(torch.as_tensor(np.fft.rfft2(phis), device="cuda"), 7)
    assert float((pp_map - pp_four).norm() / pp_map.norm()) < 1e-6
    ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    a = plan.lense_flow_pp(ft, pp_map, 7)
    b = plan.lense_flow_pp(ft, pp_four, 7)
    assert float((a - b).norm() / a.norm()) < 1e-6


def test_host_pipeline_float64_plan(torch_cuda):
    """A float64 plan's pipeline keeps the derivative-plane path and equals the device call bit for bit."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(64, 3.0, 1, B=4, seed0=61)
    plan = engine.get_plan(64, 1, R.pix_width_of(3.0), "f64")
    pipe = engine.HostPipeline(plan, 4, chunks=2)
    assert not pipe.use_pp
    fh = torch.from_numpy(f).pin_memory()
    ph = torch.from_numpy(phis).pin_memory()
    oh = torch.empty_like(fh).pin_memory()
    for _ in range(3):  # eager, capture, replay
        pipe(fh, ph, oh, n=7)
    ref = plan.lense_flow(torch.as_tensor(f, device="cuda"), plan.phi_planes(torch.as_tensor(phis, device="cuda")),
                          n=7)
    assert torch.equal(oh, ref.cpu())


def test_dlpack_entry_point(torch_cuda):
    """engine.lense_flow_dlpack takes any DLPack producer (here a numpy host array and a torch CUDA tensor)
    and returns a DLPack-capable tensor equal to the plain device call."""
    import torch
    from cmblensing_b200 import engine
    f, phis = _inputs(64, 3.0, 2, B=2, seed0=70)
    pw = R.pix_width_of(3.0)
    out = engine.lense_flow_dlpack(np.ascontiguousarray(f), torch.as_tensor(phis, device="cuda"), pw, n=7)
    assert out.is_cuda and hasattr(out, "__dlpack__")
    ref = engine.lense_flow_batch(torch.as_tensor(f, device="cuda"), torch.as_tensor(phis, device="cuda"), pw, n=7)
    assert torch.equal(out, ref)
    back = torch.from_dlpack(out.__dlpack__())
    assert back.data_ptr() == out.data_ptr()
