"""Host logic of the serving engine without a GPU: admission against slots
and the memory budget, first-fit order, arrival times, the context pool,
packing of small requests into shared batch launches, and the summary."""
import threading
import time

import numpy as np

from molspin_b200 import serving as SV
from molspin_b200 import systems as S


class FakeCtx:
    """Stands in for a device context: records its budget and whether it was closed."""
    def __init__(self, budget):
        self.budget = budget
        self.closed = False
        self.served = 0

    def close(self):
        self.closed = True


class FakeEngine(SV.ServingEngine):
    """Per-request contexts only (packing off unless asked for)."""
    def __init__(self, *a, work_s=0.05, **k):
        k.setdefault("pack_dim", 0)
        super().__init__(*a, **k)
        self.work_s = work_s
        self.active = 0
        self.peak_active = 0
        self.lock = threading.Lock()
        self.started = []
        self.ctxs = []

    def solve_pooled(self, req, budget, ctx):
        with self.lock:
            if ctx is None:
                ctx = FakeCtx(budget)
                self.ctxs.append(ctx)
            assert not ctx.closed
            ctx.served += 1
            self.active += 1
            self.peak_active = max(self.peak_active, self.active)
            self.started.append(req.rid)
        time.sleep(self.work_s)
        with self.lock:
            self.active -= 1
        return np.array([float(req.rid)]), ctx


def _reqs(n, arrivals, nuclei=(6, 7)):
    return [SV.Request(i, float(arrivals[i]), S.serving_request(i, nuclei=nuclei, steps=10), seed=i) for i in range(n)]


def test_slots_limit_concurrency_and_all_complete():
    reqs = _reqs(10, np.zeros(10))
    eng = FakeEngine(hbm_budget=1 << 40, slots=3)
    res = eng.serve(reqs, realtime=False)
    assert [r.yields[0] for r in res] == list(range(10))
    assert eng.peak_active <= 3 and eng.max_concurrency == 3
    s = SV.summarize(res)
    assert s["completed"] == 10 and s["p99_latency_s"] >= s["p50_latency_s"] > 0


def test_budget_first_fit():
    reqs = _reqs(6, np.zeros(6))
    sizes = [SV.footprint(r.workload) for r in reqs]
    budget = max(sizes) + min(sizes)
    eng = FakeEngine(hbm_budget=budget, slots=6)
    res = eng.serve(reqs, realtime=False)
    assert all(not r.error for r in res)
    assert eng.peak_reserved <= budget
    assert eng.max_concurrency >= 1


def test_oversized_request_is_refused_others_run():
    reqs = _reqs(3, np.zeros(3))
    sizes = [SV.footprint(r.workload) for r in reqs]
    eng = FakeEngine(hbm_budget=sorted(sizes)[1], slots=2)
    res = eng.serve(reqs, realtime=False)
    big = int(np.argmax(sizes))
    assert res[big].error and all(not r.error for i, r in enumerate(res) if i != big)


def test_realtime_arrivals_are_honoured():
    arrivals = np.array([0.0, 0.15, 0.3])
    reqs = _reqs(3, arrivals)
    eng = FakeEngine(hbm_budget=1 << 40, slots=4, work_s=0.01)
    res = eng.serve(reqs, realtime=True)
    for r, a in zip(res, arrivals):
        assert r.admitted >= a - 1e-3
        assert r.latency < 0.1


def test_poisson_arrivals_rate():
    a = SV.poisson_arrivals(20000, 50.0, seed=1)
    assert abs(len(a) / a[-1] - 50.0) < 2.0 and np.all(np.diff(a) > 0)


def test_footprint_grows_with_dimension():
    small = SV.footprint(S.serving_request(0, nuclei=(6, 6), steps=10))
    big = SV.footprint(S.serving_request(0, nuclei=(12, 12), steps=10))
    assert big > 10 * small


def test_contexts_are_pooled_by_shape_and_closed_at_the_end():
    # ten requests of one shape through two slots: contexts are reused, never
    # more of them than slots, and all are closed when the stream ends
    reqs = [SV.Request(i, 0.0, S.serving_request(0, nuclei=(7, 7), steps=10), seed=i) for i in range(10)]
    eng = FakeEngine(hbm_budget=1 << 40, slots=2, work_s=0.01)
    res = eng.serve(reqs, realtime=False)
    assert all(not r.error for r in res)
    assert eng.contexts_created == len(eng.ctxs) <= 2 and eng.contexts_reused == 10 - eng.contexts_created
    assert sum(c.served for c in eng.ctxs) == 10 and all(c.closed for c in eng.ctxs)
    assert eng._reserved == 0


def test_idle_contexts_are_evicted_when_memory_is_needed():
    # a small-shape context left idle must give way to a large request that
    # would not fit beside it
    small = SV.Request(0, 0.0, S.serving_request(0, nuclei=(6, 6), steps=10), seed=0)
    large = SV.Request(1, 0.05, S.serving_request(1, nuclei=(9, 9), steps=10), seed=1)
    fs, fl = SV.footprint(small.workload), SV.footprint(large.workload)
    eng = FakeEngine(hbm_budget=fl + fs // 2, slots=2, work_s=0.01)
    res = eng.serve([small, large], realtime=True)
    assert all(not r.error for r in res), [r.error for r in res]
    assert eng.peak_reserved <= eng.budget
    assert eng.ctxs[0].closed and eng.contexts_created == 2


class FakeBatch:
    def __init__(self):
        self.closed = False
        self.runs = 0

    def close(self):
        self.closed = True


class FakePackEngine(FakeEngine):
    """Packing on: solve_pack records each pack instead of launching it."""
    def __init__(self, *a, **k):
        k.setdefault("pack_dim", 2048)
        super().__init__(*a, **k)
        self.packs_seen = []
        self.batches = []

    def solve_pack(self, reqs, batch):
        with self.lock:
            if batch is None:
                batch = FakeBatch()
                self.batches.append(batch)
            assert not batch.closed
            batch.runs += 1
            self.packs_seen.append([q.rid for q in reqs])
        time.sleep(self.work_s)
        return [np.array([float(q.rid)]) for q in reqs], batch


def _small(i, steps=10, arrival=0.0):
    return SV.Request(i, arrival, S.serving_request(i, nuclei=(6, 7), steps=steps), seed=i)


def test_small_requests_share_pack_launches():
    # ten small requests at once through two slots, at most four per pack: every
    # request completes with its own result, in packs of one key, on pooled batches
    reqs = [_small(i) for i in range(10)]
    eng = FakePackEngine(hbm_budget=1 << 40, slots=2, pack_max=4, work_s=0.02)
    res = eng.serve(reqs, realtime=False)
    assert all(not r.error for r in res)
    assert [r.yields[0] for r in res] == list(range(10))
    assert sorted(i for p in eng.packs_seen for i in p) == list(range(10))
    assert all(len(p) <= 4 for p in eng.packs_seen) and len(eng.packs_seen) >= 3
    assert eng.packs == len(eng.packs_seen) and eng.packed == 10
    assert len(eng.batches) <= 2 and all(b.closed for b in eng.batches)
    assert eng.ctxs == [] and eng._reserved == 0
    assert eng.max_concurrency <= 2 * 4


def test_packs_hold_one_time_grid_and_large_requests_keep_their_contexts():
    # two step counts (two time grids) and one system above the packing
    # dimension: packs never mix grids; the large request runs on a context
    reqs = [_small(i, steps=10 if i % 2 else 20) for i in range(6)]
    reqs.append(SV.Request(6, 0.0, S.serving_request(6, nuclei=(9, 9), steps=10), seed=6))  # D = 2048
    eng = FakePackEngine(hbm_budget=1 << 40, slots=4, work_s=0.01)
    res = eng.serve(reqs, realtime=False)
    assert all(not r.error for r in res)
    steps = {q.rid: q.workload.steps for q in reqs}
    for p in eng.packs_seen:
        assert len({steps[i] for i in p}) == 1
    assert 6 not in {i for p in eng.packs_seen for i in p}
    assert sum(c.served for c in eng.ctxs) == 1 and eng.started == [6]


def test_packs_shrink_to_the_budget():
    # a budget of three of the largest footprints, below four of the smallest:
    # no pack holds more than three
    reqs = [_small(i) for i in range(7)]
    sizes = [SV.footprint(q.workload) for q in reqs]
    assert 4 * min(sizes) > 3 * max(sizes)
    eng = FakePackEngine(hbm_budget=3 * max(sizes), slots=4, work_s=0.01)
    res = eng.serve(reqs, realtime=False)
    assert all(not r.error for r in res)
    assert eng.peak_reserved <= eng.budget
    assert all(len(p) <= 3 for p in eng.packs_seen)


def test_pooled_batch_reservation_grows_with_a_larger_pack():
    # one slot: a pack of two, then (arriving later) a pack of four on the same
    # pooled batch; its reservation grows to the larger pack's footprint and is
    # returned when the stream ends
    first = [_small(i, arrival=0.0) for i in range(2)]
    later = [_small(i, arrival=0.2) for i in range(2, 6)]
    eng = FakePackEngine(hbm_budget=1 << 40, slots=1, work_s=0.05)
    res = eng.serve(first + later, realtime=True)
    assert all(not r.error for r in res)
    assert eng.packs_seen == [[0, 1], [2, 3, 4, 5]]
    assert len(eng.batches) == 1 and eng.batches[0].runs == 2 and eng.batches[0].closed
    assert eng.contexts_created == 1 and eng.contexts_reused == 1
    four = sum(SV.footprint(q.workload) for q in later)
    assert eng.peak_reserved == max(four, sum(SV.footprint(q.workload) for q in first))
    assert eng._reserved == 0
