"""Host logic of the serving loop (admission in arrival order against the HBM budget,
polling, latency accounting), driven by a fake device context: no GPU."""
import numpy as np

from radiant_b200._abi import RB_ERR_BUDGET, RadiantError
from radiant_b200 import serving as S


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeCtx:
    """Each request needs `size` bytes for `dur` seconds of device time."""

    def __init__(self, clock, budget):
        self.clock, self.budget, self.used = clock, budget, 0
        self.running = {}
        self.order = []
        self.next = 1

    def submit(self, pack):
        size, dur = pack.tables["size"], pack.tables["dur"]
        if self.used + size > self.budget:
            raise RadiantError(RB_ERR_BUDGET, "over budget")
        self.used += size
        h = self.next
        self.next += 1
        self.running[h] = (self.clock() + dur, size)
        self.order.append(pack.tables["rid"])
        return h

    def poll(self, h, rb):
        end, size = self.running[h]
        if self.clock() < end:
            return False
        self.used -= size
        del self.running[h]
        return True


class _Pack:
    def __init__(self, tables):
        self.tables = tables


def test_admission_in_arrival_order_within_budget(monkeypatch):
    clock = FakeClock()
    monkeypatch.setattr(S, "PackedProblem", _Pack)
    monkeypatch.setattr(S, "ResultBuffers", lambda p: object())
    ctx = FakeCtx(clock, budget=10)
    arr = [0.0, 0.001, 0.002, 0.003, 0.004]
    sizes = [6, 6, 2, 3, 10]
    reqs = [S.Request(i, {"size": sizes[i], "dur": 0.01, "rid": i}, arr[i]) for i in range(5)]
    loop = S.ServingLoop(ctx, poll_interval=1e-4, clock=clock, sleep=clock.sleep)
    loop.run(reqs)
    assert ctx.order == [0, 1, 2, 3, 4]          # request 1 waited for 0; 2 and 3 stayed behind 1
    assert all(r.finished is not None for r in reqs)
    assert reqs[1].submitted >= reqs[0].finished  # head-of-line wait for memory
    assert ctx.used == 0
    s = S.latency_summary(reqs)
    assert s["p99_ms"] >= s["p50_ms"] > 0 and s["requests"] == 5


def test_requests_overlap_when_they_fit(monkeypatch):
    clock = FakeClock()
    monkeypatch.setattr(S, "PackedProblem", _Pack)
    monkeypatch.setattr(S, "ResultBuffers", lambda p: object())
    ctx = FakeCtx(clock, budget=100)
    reqs = [S.Request(i, {"size": 1, "dur": 0.05, "rid": i}, 0.001 * i) for i in range(8)]
    S.ServingLoop(ctx, poll_interval=1e-4, clock=clock, sleep=clock.sleep).run(reqs)
    # all eight were on the device at once: the last finishes ~0.05 s after its arrival
    assert max(r.finished for r in reqs) < 0.007 + 0.05 + 0.001


def test_poisson_arrivals_are_seeded_and_increasing():
    a = S.poisson_arrivals(100, 50.0, 3)
    b = S.poisson_arrivals(100, 50.0, 3)
    assert np.array_equal(a, b) and np.all(np.diff(a) > 0)
    assert 1.0 < a[-1] < 3.5
