"""Continuous-batching server: results are the same alone and in the mix,
admission respects the HBM budget, and the summary reports latency."""
import numpy as np
import pytest

from openturbine_b200 import workloads as W
from openturbine_b200.serving import Request, StepServer, poisson_requests, request_pool

pytestmark = pytest.mark.gpu


def _clone(r: Request) -> Request:
    return Request(r.rid, r.kind, r.packed, r.nodes, r.steps, r.amp, r.freq, r.omega, r.roots,
                   r.arrival)


@pytest.fixture(scope="module")
def pool():
    return request_pool(16, 2, first_id=8_100_000)


def _serve(reqs, budget=0, max_active=None, precision=0):
    from openturbine_b200.runtime import Context
    ctx = Context(0, budget)
    p = W.batch_params()
    p.precision = precision
    srv = StepServer(ctx, p, max_active=max_active)
    for r in reqs:
        srv.submit(r)
    srv.run(until_s=30.0, drain=True)
    out = {r.rid: r for r in srv.finished}
    summ = srv.summary()
    ctx.close()
    return out, summ


@pytest.mark.parametrize("precision", [0, 1])
def test_same_alone_and_in_the_mix(pool, precision):
    beams, rotors = pool
    reqs = poisson_requests(200.0, 0.1, beams, rotors, rotor_fraction=0.2, steps_lo=5, steps_hi=25,
                            seed=11)
    assert any(r.kind == "rotor" for r in reqs) and len(reqs) >= 8
    mixed, summ = _serve([_clone(r) for r in reqs], precision=precision)
    assert len(mixed) == len(reqs)
    assert summ["max_active"] > 1
    for r in reqs:
        alone, _ = _serve([_clone(r)], precision=precision)
        a, b = alone[r.rid], mixed[r.rid]
        assert a.statuses == b.statuses and a.done == b.done == r.steps
        assert np.array_equal(a.final_q, b.final_q, equal_nan=True), r.rid


def test_admission_by_hbm_budget(pool):
    from openturbine_b200.runtime import Context
    beams, _ = pool
    probe = Context(0)
    mid = probe.create_model(beams[0][0])
    one = probe.used_bytes
    probe.destroy_model(mid)
    probe.close()
    # every pooled beam fits one at a time; the budget holds a few of the biggest
    sizes = []
    for packed, _ in beams:
        c = Context(0)
        c.create_model(packed)
        sizes.append(c.used_bytes)
        c.close()
    budget = int(3.5 * max(sizes))
    reqs = [Request(i, "beam", beams[i % len(beams)][0], beams[i % len(beams)][1], 6 + i % 5,
                    amp=1e4, freq=1.0, arrival=0.0) for i in range(12)]
    out, summ = _serve([_clone(r) for r in reqs], budget=budget)
    assert len(out) == 12
    assert 1 <= summ["max_active"] <= 3 + int(3.5 * max(sizes) // min(sizes))
    assert one > 0
    for r in reqs[:3]:
        alone, _ = _serve([_clone(r)])
        assert np.array_equal(alone[r.rid].final_q, out[r.rid].final_q, equal_nan=True)


def test_summary_reports_latency(pool):
    beams, rotors = pool
    reqs = poisson_requests(300.0, 0.05, beams, rotors, steps_lo=3, steps_hi=6, seed=5)
    _, summ = _serve(reqs)
    assert summ["iterations"] > 0
    assert summ["step_latency_ms"]["p99"] >= summ["step_latency_ms"]["p50"] > 0
    assert summ["beam_steps_total"] >= summ["beam_steps_converged"] > 0
