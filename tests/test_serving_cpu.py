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


def test_multi_solve_request_finishes_with_its_last_solve(monkeypatch):
    """A request of three particle solves: each solve is admitted as memory allows, and the
    request's latency ends when the last of them is collected."""
    clock = FakeClock()
    monkeypatch.setattr(S, "PackedProblem", _Pack)
    monkeypatch.setattr(S, "ResultBuffers", lambda p: object())
    ctx = FakeCtx(clock, budget=10)
    parts = [{"size": 4, "dur": 0.01, "rid": 0}, {"size": 4, "dur": 0.03, "rid": 1}, {"size": 4, "dur": 0.02, "rid": 2}]
    reqs = [S.Request(0, parts, 0.0), S.Request(1, {"size": 1, "dur": 0.01, "rid": 3}, 0.001)]
    S.ServingLoop(ctx, poll_interval=1e-4, clock=clock, sleep=clock.sleep).run(reqs)
    assert ctx.order == [0, 1, 2, 3]        # the third solve waited for memory; request 1 behind it
    assert reqs[0].finished >= 0.03 and isinstance(reqs[0].result, list) and len(reqs[0].result) == 3
    assert reqs[1].submitted >= 0.01
    s = S.latency_summary(reqs)
    assert s["requests"] == 2 and s["solves"] == 4


def test_c5_stream_draws_the_configuration():
    from radiant_b200 import workloads as W

    reqs = W.c5_stream(12, seed=2024, max_cells=300, max_groups=20, max_side=40)
    assert len(reqs) == 12
    for parts in reqs:
        assert [t["particle"] for t in parts] in (["photon"], ["photon", "electron", "positron"])
        ng = parts[0]["ng"]
        assert 10 <= ng <= 20 and all(t["ng"] == ng for t in parts)
        assert parts[0]["solver_type"] == 1 and all(t["solver_type"] == 2 for t in parts[1:])
        if parts[0]["ndims"] == 2:
            assert 32 <= parts[0]["ns"][0] <= 40 and parts[0]["nd"] in (24, 48, 80, 120, 168)
        else:
            assert 50 <= parts[0]["ns"][0] <= 300 and parts[0]["nd"] in (8, 16, 32, 64)
    # a log-uniform beam energy lands in the group that holds it
    eb, _, _ = W.log_groups(40, 20.0, 0.001)
    assert eb[W._beam_group(eb, 1.0)] >= 1.0 > eb[W._beam_group(eb, 1.0) + 1]
