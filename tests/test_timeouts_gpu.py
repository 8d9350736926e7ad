"""Device-wait timeouts are reported, not swallowed.

Every kernel block that stages its operands with bulk copies waits for them
on an mbarrier with a bounded number of polls.  Here the test hook
lf_set_wait_polls(0) makes every block's first wait run out at once, while
its copies are still legitimately in flight (nothing faults or hangs: the
drain wait that follows keeps its full limit and the copies land).  The
record must then surface: engine.wait_timeouts() reads it after a device
synchronisation, engine.check_timeouts() raises LF_ERR_TIMEOUT, every later
entry point refuses to compute (sticky), and a reset restores normal,
correct operation.
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


@pytest.mark.parametrize("N,C,adjoint", [(128, 1, False), (512, 2, False), (512, 2, True)])
def test_timed_out_wait_is_reported(torch_cuda, N, C, adjoint):
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import lens_batch
    lib = nat.load()
    theta = 2.0 if N == 512 else 3.0
    pw = R.pix_width_of(theta)
    f, phis = lens_batch(N, theta, 1, C, seed0=31)
    plan = engine.get_plan(N, C, pw)
    ft = torch.as_tensor(f, device="cuda", dtype=torch.float32)
    planes = plan.phi_planes(torch.as_tensor(phis, device="cuda"))
    good = plan.lense_flow(ft, planes, n=7, adjoint=adjoint)
    torch.cuda.synchronize()
    assert engine.wait_timeouts(reset=True) == 0
    try:
        nat.check(lib.lf_set_wait_polls(0), "lf_set_wait_polls")
        plan.lense_flow(ft, planes, n=7, adjoint=adjoint)  # queued before any block has run: returns LF_OK
        torch.cuda.synchronize()
        assert engine.wait_timeouts() == 1
        with pytest.raises(nat.LenseFlowError) as e:
            engine.check_timeouts()
        assert e.value.status == nat.LF_ERR_TIMEOUT
        # sticky: later calls refuse to compute until the record is reset
        with pytest.raises(nat.LenseFlowError) as e:
            plan.lense_flow(ft, planes, n=7, adjoint=adjoint)
        assert e.value.status == nat.LF_ERR_TIMEOUT
        assert lib.lf_stream_check(None) == nat.LF_ERR_TIMEOUT
    finally:
        nat.check(lib.lf_set_wait_polls(-1), "lf_set_wait_polls")
        engine.wait_timeouts(reset=True)
    assert lib.lf_timeout_status() == nat.LF_OK
    again = plan.lense_flow(ft, planes, n=7, adjoint=adjoint)
    torch.cuda.synchronize()
    assert engine.wait_timeouts() == 0
    assert lib.lf_stream_check(None) == nat.LF_OK
    assert torch.equal(again, good)


def test_host_pipeline_raises_on_timeout(torch_cuda):
    """The pipelined host-buffer call surfaces a timeout at its synchronisation point."""
    torch = torch_cuda
    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import lens_batch
    lib = nat.load()
    f, phis = lens_batch(128, 3.0, 4, 2, seed0=33)
    plan = engine.get_plan(128, 2, R.pix_width_of(3.0))
    pipe = engine.HostPipeline(plan, 4, chunks=2, use_graphs=False)
    fh = torch.from_numpy(f).pin_memory()
    ph = torch.from_numpy(phis).pin_memory()
    oh = torch.empty_like(fh).pin_memory()
    pipe(fh, ph, oh, n=7)
    engine.wait_timeouts(reset=True)
    try:
        nat.check(lib.lf_set_wait_polls(0), "lf_set_wait_polls")
        with pytest.raises(nat.LenseFlowError) as e:
            pipe(fh, ph, oh, n=7, wait=False)
            pipe.wait()
        assert e.value.status == nat.LF_ERR_TIMEOUT
    finally:
        nat.check(lib.lf_set_wait_polls(-1), "lf_set_wait_polls")
        torch.cuda.synchronize()
        engine.wait_timeouts(reset=True)
    pipe._pending.clear()
    pipe(fh, ph, oh, n=7)
    ref = plan.lense_flow_pp(torch.as_tensor(f, device="cuda"), plan.phi_pp(torch.as_tensor(phis, device="cuda"), 7), 7)
    assert rel_l2(oh.numpy(), ref.cpu().numpy()) == 0.0
