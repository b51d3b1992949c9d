"""GPU test of the served request loop: requests of both kinds and different
sizes share the device (pressure requests batched in one graph, viscosity
requests concurrent on their own streams, admission by a memory budget), and
each request's result is the same as when it is served alone: bit-identical
for the pressure solves (the batched graph reproduces the standalone solve)
and for the viscosity solves (independent solves on their own streams)."""
import numpy as np
import pytest

from uaamg_b200.serve import DeviceBackend, Request, Scheduler, latency_summary

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


def _stream():
    spec = [("poisson", 32, 3, 0.0), ("poisson", 48, 2, 0.0), ("viscosity", 32, 2, 0.0),
            ("poisson", 24, 1, 0.002), ("poisson", 40, 3, 0.004), ("viscosity", 24, 1, 0.004),
            ("poisson", 56, 2, 0.006)]
    return [Request(rid=i, kind=k, side=s, seed=1000 + 17 * i, substeps=n, arrival=a)
            for i, (k, s, n, a) in enumerate(spec)]


def _serve(reqs, batching=True, budget=None):
    be = DeviceBackend(batching=batching, keep_results=True)
    sch = Scheduler(be, budget if budget is not None else 40 * 10 ** 9)
    sch.run(reqs, time_limit=600.0)
    assert len(sch.done) == len(reqs)
    return sch, be


def test_served_results_same_alone_and_in_the_mix(gpu):
    mix = _stream()
    sch, be = _serve(mix)
    assert sch.rounds >= 3 and be.batch_builds >= 1
    for r in mix:
        assert len(r.iterations) == r.substeps and all(s == 0 for s in r.status), (r.rid, r.status)
    for r in mix:
        alone = Request(rid=r.rid, kind=r.kind, side=r.side, seed=r.seed, substeps=r.substeps, arrival=0.0)
        _serve([alone])
        assert np.array_equal(alone.result, r.result), r.rid
        assert alone.iterations == r.iterations, (r.rid, alone.iterations, r.iterations)
    s = latency_summary(sch.done)
    assert s["p99_ms"] >= s["p50_ms"] > 0


def test_plain_form_and_tight_budget_give_the_same_results(gpu):
    mix = _stream()
    _serve(mix)
    plain = _stream()
    _serve(plain, batching=False)
    tight = _stream()
    one = DeviceBackend.estimate_bytes(max(tight, key=lambda r: DeviceBackend.estimate_bytes(r)))
    sch, _ = _serve(tight, budget=one)  # at most one large request resident at a time
    assert sch.peak_used <= one
    for a, b, c in zip(mix, plain, tight):
        assert np.array_equal(a.result, b.result) and np.array_equal(a.result, c.result), a.rid
        assert a.iterations == b.iterations == c.iterations
