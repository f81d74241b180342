"""Serving loop: continuous batching of SN solve requests over rb_submit / rb_poll.

Requests arrive over time (for instance as a seeded Poisson stream). A request holds one or
more particle solves (a photon solve alone, or photon, electron and positron solves of one
case). Each solve of an arrived request is admitted as soon as its device state fits the
context's HBM budget; admission keeps arrival order (a solve that does not fit holds the ones
behind it, so large requests are not starved). An admitted solve is launched at once on its own
stream, beside the solves already on the device (rb_submit); finished ones are collected by
polling, which also frees their memory for the next admissions. A request's latency runs from
its arrival to the moment the results of all its solves are back in host memory.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from ._abi import RB_ERR_BUDGET, PackedProblem, RadiantError, ResultBuffers


@dataclass
class Request:
    rid: int
    tables: dict | list                 # one solve's tables, or the list of a request's solves
    arrival: float                      # seconds after the start of the run
    submitted: float | None = None      # when its first solve was admitted
    finished: float | None = None       # when its last solve's results were back
    result: ResultBuffers | list | None = None  # ResultBuffers (one solve) or one per solve
    _packs: list = field(default_factory=list, repr=False)
    _results: list = field(default_factory=list, repr=False)
    _next: int = field(default=0, repr=False)   # next solve to admit
    _open: int = field(default=0, repr=False)   # solves admitted and not yet collected

    @property
    def parts(self) -> list:
        return self.tables if isinstance(self.tables, list) else [self.tables]

    @property
    def results(self) -> list:
        return self.result if isinstance(self.result, list) else [self.result]

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class ServingLoop:
    """Drives a Context (or any object with submit / poll of the same meaning)."""

    def __init__(self, ctx, poll_interval: float = 50e-6, clock=time.perf_counter, sleep=time.sleep):
        self.ctx = ctx
        self.poll_interval = poll_interval
        self.clock = clock
        self.sleep = sleep

    def run(self, requests: list[Request], timeout: float = 600.0) -> list[Request]:
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        inflight: dict[int, tuple[Request, int]] = {}
        t0 = self.clock()
        i = 0
        while i < len(pending) or inflight:
            now = self.clock() - t0
            if now > timeout:
                raise TimeoutError(f"serving run exceeded {timeout} s with {len(inflight)} solves in flight")
            progressed = False
            # admit in arrival order, solve by solve, while the budget allows
            while i < len(pending) and pending[i].arrival <= now:
                req = pending[i]
                if not req._packs:
                    req._packs = [PackedProblem(t) for t in req.parts]
                    req._results = [ResultBuffers(p) for p in req._packs]
                    req.result = req._results if isinstance(req.tables, list) else req._results[0]
                blocked = False
                while req._next < len(req._packs):
                    try:
                        h = self.ctx.submit(req._packs[req._next])
                    except RadiantError as e:
                        if e.status == RB_ERR_BUDGET and inflight:
                            blocked = True  # wait for memory to free up
                            break
                        raise
                    if req.submitted is None:
                        req.submitted = self.clock() - t0
                    inflight[h] = (req, req._next)
                    req._next += 1
                    req._open += 1
                    progressed = True
                if blocked:
                    break
                i += 1
            # collect finished solves
            for h in list(inflight):
                req, k = inflight[h]
                if self.ctx.poll(h, req._results[k]):
                    del inflight[h]
                    req._open -= 1
                    if req._open == 0 and req._next == len(req._packs):
                        req.finished = self.clock() - t0
                    progressed = True
            if not progressed:
                self.sleep(self.poll_interval)
        return requests


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times (s) of a Poisson stream of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def latency_summary(requests: list[Request]) -> dict:
    lat = np.array([r.latency for r in requests])
    span = max(r.finished for r in requests) - min(r.arrival for r in requests)
    nsolves = sum(len(r.parts) for r in requests)
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "requests_per_s": len(requests) / span,
            "solves_per_s": nsolves / span, "requests": len(requests), "solves": nsolves}
