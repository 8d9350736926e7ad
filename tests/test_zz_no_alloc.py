"""The allocation-free entry point lf_lense_flow_noalloc, called through the C ABI.

Some callers cannot allocate device memory: a framework that has reserved
nearly all of the GPU's memory for its own pool (where one more cudaMalloc
can fail), or a latency-critical loop where cudaMalloc/cudaFree would
synchronise the device.  lf_lense_flow_noalloc serves them with scratch held
in a fixed-size device array inside the library.  These tests check it
against the allocating entry point lf_lense_flow on two calls in a row (so
the second call runs on scratch left over from the first), and that an
oversized request is refused.  The file is named so that pytest collects it
last.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL32 = 1e-5  # the FP32 engine's parity tolerance


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _call_noalloc(lib, torch, N, C, pw, f, out, planes, B, n, direction, adjoint):
    from cmblensing_b200 import _native as nat
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = lambda t: nat.LF_F64 if t.dtype == torch.float64 else nat.LF_F32
    return lib.lf_lense_flow_noalloc(N, C, ctypes.c_double(pw), ctypes.c_void_p(f.data_ptr()), code(f),
                                     ctypes.c_void_p(out.data_ptr()), code(out), ctypes.c_void_p(planes.data_ptr()),
                                     B, n, direction, int(adjoint), stream)


# (N, C, batch, theta): every component count, and twiddle offsets into the shared tables for 64, 256 and 512;
# the largest needs 5 x 4 x 512^2 x 3 bytes = 15 MiB of the 24 MiB scratch
SHAPES = [(256, 2, 2, 3.0), (64, 1, 2, 3.0), (512, 3, 1, 2.0)]


@pytest.mark.parametrize("N,C,B,theta", SHAPES)
def test_noalloc_matches_allocating_entry_point_twice(torch_cuda, N, C, B, theta):
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import lens_batch, ARCMIN
    lib = nat.load()
    pw = theta * ARCMIN
    plan = engine.get_plan(N, C, pw)
    # call 1: forward lens; call 2: adjoint lens of other maps, on the scratch the first call left behind
    cases = [(0, 1, False), (10, 1, True)]
    for seed0, direction, adjoint in cases:
        f, phis = lens_batch(N, theta, B, C, seed0=seed0)
        ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
        planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
        out = torch.empty_like(ft)
        status = _call_noalloc(lib, torch, N, C, pw, ft, out, planes, B, 7, direction, adjoint)
        assert status == nat.LF_OK, nat.status_string(status)
        ref = plan.lense_flow(ft, planes, n=7, direction=direction, adjoint=adjoint)
        torch.cuda.synchronize()
        assert rel_l2(out.double().cpu().numpy(), ref.double().cpu().numpy()) < TOL32


def test_noalloc_float64_in_place_inverse(torch_cuda):
    """float64 fields in and out, f_in == f_out (an in-place inverse lens), against the allocating entry point."""
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import lens_batch, ARCMIN
    lib = nat.load()
    N, C, B, theta = 128, 2, 3, 3.0
    pw = theta * ARCMIN
    plan = engine.get_plan(N, C, pw)
    f, phis = lens_batch(N, theta, B, C, seed0=21)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    x = torch.as_tensor(f, device="cuda")  # float64
    ref = plan.lense_flow(x, planes, n=7, direction=-1)
    for _ in range(2):
        y = x.clone()
        status = _call_noalloc(lib, torch, N, C, pw, y, y, planes, B, 7, -1, False)
        assert status == nat.LF_OK, nat.status_string(status)
        torch.cuda.synchronize()
        assert y.dtype == torch.float64
        assert rel_l2(y.cpu().numpy(), ref.cpu().numpy()) < TOL32


def test_noalloc_zero_steps_needs_no_scratch(torch_cuda):
    """nsteps = 0 returns the input (as lf_lense_flow does), even for a size beyond the scratch."""
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    lib = nat.load()
    N, C, B = 1024, 3, 1
    f = torch.randn((B, C, N, N), device="cuda")
    out = torch.empty_like(f)
    planes = torch.zeros((B, 5, N, N), device="cuda")
    assert _call_noalloc(lib, torch, N, C, 1e-3, f, out, planes, B, 0, 1, False) == nat.LF_OK
    torch.cuda.synchronize()
    assert torch.equal(out, f)


def test_noalloc_rejects_requests_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    lib = nat.load()
    N, C, B = 1024, 3, 1  # needs 16 x 1024^2 x 3 bytes > 24 MiB
    assert 16 * N * N * C * B > nat.LF_NOALLOC_SCRATCH_BYTES
    f = torch.zeros((B, C, N, N), device="cuda")
    planes = torch.zeros((B, 5, N, N), device="cuda")
    status = _call_noalloc(lib, torch, N, C, 1e-3, f, f, planes, B, 7, 1, False)
    assert status == nat.LF_ERR_WORKSPACE
    assert "workspace" in nat.status_string(status)
