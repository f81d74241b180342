"""Serving loop: continuous batching of SN solve requests over rb_submit / rb_poll.

Requests arrive over time (for instance as a seeded Poisson stream). Each arrived request is
admitted as soon as its device state fits the context's HBM budget; admission keeps arrival
order (a request that does not fit holds the ones behind it, so large requests are not
starved). Admitted requests run at once, beside the ones already on the device; finished ones
are collected by polling, which also frees their memory for the next admissions. Latency is
measured from arrival to the moment the result is back in host memory.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from ._abi import RB_ERR_BUDGET, PackedProblem, RadiantError, ResultBuffers


@dataclass
class Request:
    rid: int
    tables: dict
    arrival: float                      # seconds after the start of the run
    submitted: float | None = None
    finished: float | None = None
    result: ResultBuffers | None = None
    _pack: PackedProblem | None = field(default=None, repr=False)

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
        inflight: dict[int, Request] = {}
        t0 = self.clock()
        i = 0
        while i < len(pending) or inflight:
            now = self.clock() - t0
            if now > timeout:
                raise TimeoutError(f"serving run exceeded {timeout} s with {len(inflight)} requests in flight")
            progressed = False
            # admit in arrival order while the budget allows
            while i < len(pending) and pending[i].arrival <= now:
                req = pending[i]
                if req._pack is None:
                    req._pack = PackedProblem(req.tables)
                    req.result = ResultBuffers(req._pack)
                try:
                    h = self.ctx.submit(req._pack)
                except RadiantError as e:
                    if e.status == RB_ERR_BUDGET and inflight:
                        break  # wait for memory to free up
                    raise
                req.submitted = self.clock() - t0
                inflight[h] = req
                i += 1
                progressed = True
            # collect finished requests
            for h in list(inflight):
                req = inflight[h]
                if self.ctx.poll(h, req.result):
                    req.finished = self.clock() - t0
                    del inflight[h]
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
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "solves_per_s": len(requests) / span, "requests": len(requests)}
