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


def test_noalloc_matches_allocating_entry_point_twice(torch_cuda):
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import lens_batch, ARCMIN
    lib = nat.load()
    N, C, theta = 256, 2, 3.0
    pw = theta * ARCMIN
    plan = engine.get_plan(N, C, pw)
    # call 1: forward lens of two maps; call 2: adjoint lens of two other maps
    cases = [(0, 1, False), (10, 1, True)]
    for seed0, direction, adjoint in cases:
        f, phis = lens_batch(N, theta, 2, C, seed0=seed0)
        ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
        planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
        out = torch.empty_like(ft)
        status = _call_noalloc(lib, torch, N, C, pw, ft, out, planes, 2, 7, direction, adjoint)
        assert status == nat.LF_OK, nat.status_string(status)
        ref = plan.lense_flow(ft, planes, n=7, direction=direction, adjoint=adjoint)
        torch.cuda.synchronize()
        assert rel_l2(out.double().cpu().numpy(), ref.double().cpu().numpy()) < TOL32


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
