"""Host-side logic of the serving layer (no GPU): batch-size buckets, latency summaries and the
per-stage breakdown of the slowest lens requests."""
import pytest

from cmblensing_b200 import serve


def _req(kind, submit, admit, launch, issued, seen):
    r = serve.Request(kind, 128, 1, 3.0)
    r.t_submit, r.t_admit, r.t_launch, r.t_issued, r.t_seen, r.t_done = submit, admit, launch, issued, seen, seen
    return r


def test_bucket_rounds_up_to_powers_of_two():
    assert [serve._bucket(b) for b in (1, 2, 3, 4, 5, 8, 9, 16)] == [1, 2, 4, 4, 8, 8, 16, 16]


def test_lens_tail_breakdown_averages_the_slowest_stages():
    # 99 fast lens requests (1 ms) and one slow one whose time splits 10 / 20 / 30 / 40 ms over the stages
    reqs = [_req("lens", 0.0, 0.0, 0.0, 0.0005, 0.001) for _ in range(99)]
    reqs.append(_req("delens", 1.0, 1.010, 1.030, 1.060, 1.100))
    reqs.append(_req("wf", 0.0, 0.0, None, None, 9.0))  # Wiener filters are not lens requests
    t = serve.lens_tail_breakdown(reqs, frac=0.01)
    assert t["n"] == 1
    assert t["latency_ms"] == pytest.approx(100.0)
    assert t["admission_ms"] == pytest.approx(10.0)
    assert t["slot_wait_ms"] == pytest.approx(20.0)
    assert t["stage_and_issue_ms"] == pytest.approx(30.0)
    assert t["gpu_until_seen_ms"] == pytest.approx(40.0)
    assert serve.lens_tail_breakdown([]) == {}


def test_latency_summary_percentiles():
    reqs = [_req("lens", 0.0, 0.0, 0.0, 0.0, 0.001 * (i + 1)) for i in range(100)]
    s = serve.latency_summary(reqs)
    assert s["n"] == 100
    assert s["p50_ms"] == pytest.approx(50.5)
    assert 99.0 <= s["p99_ms"] <= 100.0
    assert serve.latency_summary([]) == {}
