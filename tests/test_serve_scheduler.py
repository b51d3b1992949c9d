"""Host logic of the served request loop (no GPU): arrivals, admission by
memory budget, round-based continuous batching, latency accounting.  The
device work is replaced by a fake backend with a simulated clock."""
import numpy as np
import pytest

from uaamg_b200.serve import Request, Scheduler, latency_summary, make_stream


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


class FakeBackend:
    """Costs: side^3 bytes; a pressure round takes 1 ms + 0.2 ms per resident
    pressure request (batched); a viscosity lane takes 5 ms per substep and
    runs concurrently with the rounds."""

    def __init__(self, clock, budget_log):
        self.clock = clock
        self.resident = {}
        self.rounds = []
        self.lanes = {}
        self.budget_log = budget_log

    @staticmethod
    def estimate_bytes(r):
        return r.side ** 3

    def admit(self, r):
        assert r.rid not in self.resident
        self.resident[r.rid] = r

    def release(self, r):
        del self.resident[r.rid]
        self.lanes.pop(r.rid, None)

    def poisson_round(self, pois):
        assert all(r.rid in self.resident and r.kind == "poisson" for r in pois)
        self.rounds.append([r.rid for r in pois])
        for r in pois:
            r.iterations.append(5)
            r.status.append(0)
        self.budget_log.append(sum(x.side ** 3 for x in self.resident.values()))
        self.clock.t += 1e-3 + 0.2e-3 * len(pois)

    def start_viscosity(self, r):
        assert r.rid in self.resident and r.kind == "viscosity"
        self.lanes[r.rid] = self.clock.t + 5e-3 * r.substeps
        r.iterations.extend([7] * r.substeps)
        r.status.extend([0] * r.substeps)

    def viscosity_done(self, r):
        return self.clock.t >= self.lanes[r.rid]

    def wait_viscosity(self, seconds):
        self.clock.t += seconds


def test_make_stream_rates_and_determinism():
    a = make_stream(2.0, seed=3)
    b = make_stream(2.0, seed=3)
    assert [(r.kind, r.side, r.substeps, r.arrival) for r in a] == [(r.kind, r.side, r.substeps, r.arrival) for r in b]
    npois = sum(r.kind == "poisson" for r in a)
    nvisc = sum(r.kind == "viscosity" for r in a)
    assert 320 <= npois <= 480 and 60 <= nvisc <= 140  # 200/s and 50/s over 2 s
    assert all(48 <= r.side <= 384 and r.side % 8 == 0 for r in a)
    assert all(1 <= r.substeps <= 24 for r in a)
    assert all(a[i].arrival <= a[i + 1].arrival for i in range(len(a) - 1))
    assert [r.rid for r in a] == list(range(len(a)))
    sides = np.array([r.side for r in a], dtype=np.float64)
    # log-uniform on [48, 384]: the median is near sqrt(48 * 384) ~ 136
    assert 100 <= np.median(sides) <= 180


def test_every_request_served_exactly_its_substeps_within_budget():
    clock = FakeClock()
    log = []
    be = FakeBackend(clock, log)
    reqs = make_stream(0.3, seed=1)
    budget = 3 * 384 ** 3
    sch = Scheduler(be, budget)
    sch.run(reqs, clock=clock, sleep=clock.sleep, time_limit=1e9)
    assert len(sch.done) == len(reqs) and not sch.active and not sch.queue
    for r in reqs:
        assert len(r.iterations) == r.substeps == r.step
        assert r.admitted_at >= r.arrival and r.done_at > r.admitted_at
        assert r.latency > 0
    assert max(log) <= budget and sch.peak_used <= budget
    assert sch.used == 0 and not be.resident
    assert sch.solves == sum(r.substeps for r in reqs)


def test_admission_waits_for_memory_and_keeps_arrival_order():
    clock = FakeClock()
    be = FakeBackend(clock, [])
    big = [Request(rid=i, kind="poisson", side=100, seed=i, substeps=3, arrival=0.0) for i in range(3)]
    sch = Scheduler(be, budget_bytes=2 * 100 ** 3 + 10)
    for r in big:
        sch.submit(r)
    adm = sch.admit(0.0)
    assert [r.rid for r in adm] == [0, 1] and [r.rid for r in sch.queue] == [2]
    for _ in range(3):
        sch.round(clock)
    assert [r.rid for r in sch.done] == [0, 1] and sch.used == 0
    assert [r.rid for r in sch.admit(clock())] == [2]


def test_continuous_batching_joins_new_arrivals_at_the_next_round():
    clock = FakeClock()
    be = FakeBackend(clock, [])
    sch = Scheduler(be, budget_bytes=10 ** 9)
    a = Request(rid=0, kind="poisson", side=32, seed=0, substeps=4, arrival=0.0)
    b = Request(rid=1, kind="poisson", side=32, seed=1, substeps=2, arrival=0.001)
    c = Request(rid=2, kind="viscosity", side=32, seed=2, substeps=1, arrival=0.001)
    sch.run([a, b, c], clock=clock, sleep=clock.sleep, time_limit=1.0)
    # pressure round 1 holds a alone; b joins in round 2 (arrived during round
    # 1) and leaves after round 3; a leaves after round 4.  c's lane (5 ms)
    # runs beside the rounds and finishes after them.
    assert be.rounds == [[0], [0, 1], [0, 1], [0]]
    assert b.done_at < a.done_at < c.done_at
    assert c.admitted_at == pytest.approx(1.2e-3) and c.done_at >= c.admitted_at + 5e-3
    assert len(c.iterations) == 1 and c.step == 1


def test_request_larger_than_budget_is_an_error():
    clock = FakeClock()
    sch = Scheduler(FakeBackend(clock, []), budget_bytes=1000)
    sch.submit(Request(rid=0, kind="poisson", side=64, seed=0, substeps=1, arrival=0.0))
    with pytest.raises(ValueError):
        sch.admit(0.0)


def test_latency_summary():
    rs = [Request(rid=i, kind="poisson", side=8, seed=i, substeps=1, arrival=0.0, done_at=(i + 1) * 1e-3)
          for i in range(100)]
    s = latency_summary(rs)
    assert s["p50_ms"] == pytest.approx(50.5, abs=0.01) and s["max_ms"] == pytest.approx(100.0)
    assert 99.0 <= s["p99_ms"] <= 100.0
