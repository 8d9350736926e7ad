"""The continuous-batching service: every result equals the same request run alone.

Lens and delens requests are batched and replayed from captured CUDA graphs;
each map still runs the kernels and tiles it would use alone, so results
must be bit-identical.  Wiener-filter requests of one size are solved
together by the batched CG, whose inner products sum in a different order
than a solo solve: they must agree with the solo solution within the
workload's CG tolerance, 1e-6.
"""
import threading
import time

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _lens_req(kind, N, C, theta, seed):
    from cmblensing_b200.serve import Request
    from cmblensing_b200.simulate import lens_batch
    f, phis = lens_batch(N, theta, 1, C, seed0=seed)
    return Request(kind, N, C, theta, f=f[0], phi=phis[0], n=7)


def _wf_req(N, seed):
    import cmblensing_b200 as cl
    from cmblensing_b200 import matrix_operators as mo
    from cmblensing_b200.serve import Request
    from cmblensing_b200.simulate import inference_problem
    from oracle import lenseflow_ref as R
    p = inference_problem(N, 2.0, beam_fwhm=1.0, noise_t=2.0, noise_p=2.0, seed=seed, bb_fraction=0.01)
    pw = R.pix_width_of(2.0)
    kw = dict(nside=N, theta_pix=2.0, pix_width=pw, fourier_weights=R.get_fourier_weights((N, N)))
    eb = lambda a, b: mo.DiagonalEB(matrix_EE=a, matrix_BB=b, **kw)
    ones = np.ones_like(p["beam"])
    data = cl.FlatS2(polar_matrix_1=p["beam"] * p["e"] + p["n_e"], polar_matrix_2=p["n_b"], **kw)
    prob = dict(phi=cl.FlatS0(scalar_matrix=p["phi"], **kw), data=data, Cf=eb(p["cf_ee"], p["cf_bb"]),
                Cn=eb(p["cn_p"], p["cn_p"]), M=eb(ones, ones), B=eb(p["beam"], p["beam"]))
    return Request("wf", N, 2, 2.0, problem=prob, n=7, wf_kwargs=dict(rel_tol=1e-6, refine_every=10))


def test_mixed_stream_equals_solo_runs(torch_cuda):
    from cmblensing_b200.serve import Server, latency_summary, run_alone
    reqs = []
    rng = np.random.default_rng(0)
    for i in range(32):  # the workload's grid sizes
        N = [128, 256, 512, 1024][rng.integers(4)]
        C = [1, 2][rng.integers(2)]
        kind = ["lens", "delens"][rng.integers(2)]
        reqs.append(_lens_req(kind, N, C, 3.0 if N < 512 else 2.0, seed=10 * i))
    # Wiener filters of three sizes: two workers solve (and capture their CG graphs) concurrently
    reqs += [_wf_req(64, seed=s) for s in (1, 2, 3)] + [_wf_req(128, seed=4), _wf_req(512, seed=5)]
    rng.shuffle(reqs)
    srv = Server(max_batch=8, wf_workers=2).start()
    for r in reqs:
        srv.submit(r)
        time.sleep(float(rng.exponential(0.002)))
    for r in reqs:
        assert r.done.wait(120), "request timed out"
    srv.stop()
    for r in reqs:
        assert r.error is None, r.error
        alone = run_alone(r)
        if r.kind == "wf":
            for k in alone._matrix_names():
                assert rel_l2(getattr(r.result, k), getattr(alone, k)) < 1e-6
        else:
            assert np.array_equal(r.result, alone), (r.kind, r.nside, r.ncomp)
    s = latency_summary(reqs)
    assert s["n"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0


def test_tight_budget_still_completes_and_singular_phi_fails_alone(torch_cuda):
    from cmblensing_b200 import _native as nat
    from cmblensing_b200.serve import Request, Server
    from cmblensing_b200.simulate import gaussian_phi
    good = [_lens_req("lens", 128, 2, 3.0, seed=s) for s in range(5)]
    bad = _lens_req("lens", 128, 2, 3.0, seed=99)
    bad.phi = gaussian_phi(128, 3.0, seed=7, spectrum="literal")
    srv = Server(hbm_budget=1, max_batch=4).start()  # admits one request at a time
    for r in good[:2] + [bad] + good[2:]:
        srv.submit(r)
    for r in good + [bad]:
        assert r.done.wait(120)
    srv.stop()
    assert all(r.error is None for r in good)
    assert isinstance(bad.error, nat.SingularMagnificationError)


def test_prepared_slots_serve_without_new_captures(torch_cuda):
    """Server.prepare creates a shape's slots and every bucket's graph up front; serving then adds none."""
    from cmblensing_b200.serve import Server, run_alone
    srv = Server(max_batch=4, wf_workers=1).prepare(128, 2, 3.0)
    keys = sorted(srv.slots)
    assert [k[3] for k in keys] == [-1, 1] and all(len(srv.slots[k]) == 2 for k in keys)
    graphs = {k: [sorted(s.graphs) for s in srv.slots[k]] for k in keys}
    assert all(g == [1, 2, 4] for gs in graphs.values() for g in gs)
    reqs = [_lens_req(["lens", "delens"][i % 2], 128, 2, 3.0, seed=50 + i) for i in range(7)]
    srv.start()
    with pytest.raises(RuntimeError):
        srv.prepare(128, 1, 3.0)
    for r in reqs:
        srv.submit(r)
    for r in reqs:
        assert r.done.wait(120)
    srv.stop()
    assert sorted(srv.slots) == keys
    assert {k: [sorted(s.graphs) for s in srv.slots[k]] for k in keys} == graphs
    for r in reqs:
        assert r.error is None, r.error
        assert np.array_equal(r.result, run_alone(r))
