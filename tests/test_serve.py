"""The request loop's admission and continuous batching, on the CPU: a
simulated executor whose batches take (fixed + per-row) virtual seconds, and
a virtual clock the loop's idle sleeps advance."""
import pytest

from visondf_b200 import serve


class Clock:
    def __init__(self):
        self.t = 0.0

    def now(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class SimExecutor:
    def __init__(self, clock, slots=2, fixed=1e-4, per_row=1e-9):
        self.clock, self.nslots, self.fixed, self.per_row = clock, slots, fixed, per_row
        self.running = 0
        self.batches = []

    def free_slots(self, inflight):
        return inflight < self.nslots

    def start(self, reqs):
        end = self.clock.t + self.fixed + self.per_row * sum(r.rows for r in reqs)
        self.batches.append([r.rid for r in reqs])
        return (end, [r.rid for r in reqs])

    def done(self, h):
        return self.clock.t >= h[0]

    def finish(self, h):
        return list(h[1])


def trace(n=200, gap=2e-4, rows=100_000, need=1000):
    return [serve.Request(rid=i, arrival=i * gap, rows=rows, need_bytes=need) for i in range(n)]


def run(reqs, slots=2, budget=10**12, fixed=0, **kw):
    clk = Clock()
    ex = SimExecutor(clk, slots=slots)
    loop = serve.Loop(ex, budget, fixed, clock=clk.now, idle_sleep=clk.sleep, **kw)
    return loop.run(reqs), ex


def test_every_request_completes_in_arrival_order():
    reqs = trace()
    st, ex = run(reqs)
    assert st.requests == 200 and all(r.completed is not None and r.latency >= 0 for r in reqs)
    started = [r.started for r in sorted(reqs, key=lambda r: r.arrival)]
    assert started == sorted(started)  # first come, first served
    assert [rid for b in ex.batches for rid in b] == list(range(200))
    assert all(r.result == r.rid for r in reqs)


def test_budget_is_never_exceeded():
    reqs = trace(need=400)
    st, ex = run(reqs, budget=1000, fixed=100)
    assert st.max_in_flight_bytes <= 1000
    # at most two requests of 400 bytes fit beside 100 fixed bytes
    assert max(len(b) for b in ex.batches) <= 2


def test_request_larger_than_budget_is_refused():
    with pytest.raises(ValueError):
        run(trace(n=3, need=2000), budget=1000)
    with pytest.raises(ValueError):
        run(trace(n=3), budget=10, fixed=20)


def test_arrivals_join_the_next_batch_while_one_runs():
    # a burst: requests arrive faster than one batch completes
    reqs = trace(n=300, gap=1e-5, rows=1_000_000)
    st, ex = run(reqs, slots=2)
    assert st.batches < 300 / 4           # requests were batched together
    assert max(len(b) for b in ex.batches) > 4
    # a second batch started before the first one completed (overlap)
    first = [r for r in reqs if r.rid in ex.batches[0]]
    second = [r for r in reqs if r.rid in ex.batches[1]]
    assert second[0].started < first[0].completed


def test_single_slot_single_query_is_one_at_a_time():
    reqs = trace(n=50, gap=1e-5)
    st, ex = run(reqs, slots=1, max_batch_queries=1)
    assert st.batches == 50 and all(len(b) == 1 for b in ex.batches)
    order = sorted(reqs, key=lambda r: r.rid)
    for a, b in zip(order, order[1:]):
        assert b.started >= a.completed   # never overlapping


def test_batch_limits():
    reqs = trace(n=100, gap=0.0, rows=1000)
    st, ex = run(reqs, slots=1, max_batch_rows=10_000, max_batch_queries=7)
    assert max(len(b) for b in ex.batches) <= 7
    assert all(len(b) * 1000 <= 10_000 for b in ex.batches)


def test_percentile_nearest_rank():
    xs = list(range(1, 101))
    assert serve.percentile(xs, 50) == 50 and serve.percentile(xs, 99) == 99 and serve.percentile(xs, 100) == 100
    assert serve.percentile([3.0], 99) == 3.0
