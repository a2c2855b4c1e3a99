"""Serving form: continuous batching under a device-memory budget.

Each request's result in the mix must equal its solo run within 1e-12
relative (the only freedom is the SpMM tile the autotuner picks under load,
which regroups partial sums; small requests run packed in the batching form
and alone as one-system batches, bit for bit the same), admission must
respect the budget, and every request must complete.
"""
import numpy as np
import pytest

from molspin_b200 import serving as SV
from molspin_b200 import systems as S

pytestmark = pytest.mark.gpu


def _requests(n, steps, nuclei, rate=200.0):
    arr = SV.poisson_arrivals(n, rate, seed=3)
    return [SV.Request(i, float(arr[i]), S.serving_request(i, nuclei=nuclei, steps=steps), seed=1000 + i)
            for i in range(n)]


def test_mix_equals_solo_and_overlaps():
    reqs = _requests(8, 40, (6, 11))  # D = 256 .. 8192: resident and streamed forms
    eng = SV.ServingEngine(0, hbm_budget=40 << 30, slots=4)
    res = eng.serve(reqs)
    assert all(not r.error for r in res), [r.error for r in res]
    assert eng.max_concurrency >= 2
    solo = SV.ServingEngine(0, hbm_budget=40 << 30, slots=1)
    for r, q in zip(res, reqs):
        alone = solo.solve(q)
        assert np.max(np.abs(r.yields - alone)) <= 1e-12 * np.max(np.abs(alone)), r.rid
    summary = SV.summarize(res)
    assert summary["completed"] == 8 and summary["p99_latency_s"] >= summary["p50_latency_s"]


def test_small_requests_packed_into_one_launch():
    # six small requests (D = 256, 512) at once: they share pack launches of the
    # batching form; each equals its solo run (a one-system batch) bit for bit
    # and the per-request context path within the complex64 forms' 1e-6
    reqs = _requests(6, 30, (6, 7), rate=1e6)
    eng = SV.ServingEngine(0, hbm_budget=40 << 30, slots=2)
    res = eng.serve(reqs, realtime=False)
    assert all(not r.error for r in res), [r.error for r in res]
    assert eng.packed == 6 and 1 <= eng.packs < 6
    solo = SV.ServingEngine(0, hbm_budget=40 << 30, slots=1)
    ctx = SV.ServingEngine(0, hbm_budget=40 << 30, slots=1, pack_dim=0)
    for r, q in zip(res, reqs):
        np.testing.assert_array_equal(r.yields, solo.solve(q))
        alone = ctx.solve(q)
        assert np.max(np.abs(r.yields - alone)) <= 1e-6 * np.max(np.abs(alone)), r.rid


def test_admission_respects_budget():
    reqs = _requests(4, 20, (6, 8), rate=1e6)
    biggest = max(SV.footprint(q.workload) for q in reqs)
    eng = SV.ServingEngine(0, hbm_budget=biggest + (1 << 20), slots=4)
    res = eng.serve(reqs)
    assert all(not r.error for r in res), [r.error for r in res]
    assert eng.peak_reserved <= eng.budget
    # a request larger than the whole budget is refused, the others still run
    tiny = SV.ServingEngine(0, hbm_budget=1 << 20, slots=2)
    res = tiny.serve(reqs[:1])
    assert res[0].error
