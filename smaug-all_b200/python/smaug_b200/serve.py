"""Serving loop: continuous batching of simulation requests on one GPU.

No counterpart in the reference (one SMAUG process runs one simulation).
Requests (a problem and a number of RK4 steps) arrive over time.  The loop
admits them, first come first served, into one device-resident batch while
its arena has a free block of the request's footprint.  It advances every
admitted simulation together in chunks of steps (one launch per RK stage for
all of them, CUDA graphs).  After each chunk it retires the finished ones:
their state is copied to the host, their slot and memory are freed, and
waiting requests take their place.  A request's time to solution runs from
its arrival to its result on the host.

Each simulation keeps its own dt, driver clock and step budget on the device,
so a result is bit-identical to the same simulation run alone
(tests/test_gpu_serve.py checks this).
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import PREC_MIXED


@dataclass
class Request:
    rid: int
    prob: object
    nsteps: int
    arrival: float                    # seconds after the stream starts
    admitted: float | None = None
    done: float | None = None
    slot: int | None = None
    result: np.ndarray | None = field(default=None, repr=False)

    @property
    def latency(self) -> float | None:
        return None if self.done is None else self.done - self.arrival


def poisson_stream(count: int, rate: float, make, seed: int = 777, duration: float | None = None) -> list:
    """`count` requests with exponential inter-arrival gaps of mean 1/rate
    (stopping at `duration` seconds if given); make(i, rng) -> (problem, nsteps)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        if duration is not None and t > duration:
            break
        prob, nsteps = make(i, rng)
        out.append(Request(i, prob, int(nsteps), t))
    return out


class Server:
    """Runs a request stream through one batch (any object with the Batch
    methods add / step / poll / state / remove)."""

    def __init__(self, batch, chunk: int = 8, keep_results: bool = True):
        self.batch = batch
        self.chunk = chunk
        self.keep_results = keep_results

    def run(self, requests, realtime: bool = True, clock=time.perf_counter, sleep=time.sleep) -> dict:
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        queue: deque = deque()
        active: dict = {}
        i, steps_done, chunks = 0, 0, 0
        max_active = 0
        while i < len(reqs) or queue or active:
            t = now()
            while i < len(reqs) and (reqs[i].arrival <= t or not realtime):
                queue.append(reqs[i])
                i += 1
            while queue:  # first come first served: the head waits until it fits
                r = queue[0]
                slot = self.batch.add(r.prob, r.nsteps)
                if slot is None:
                    break
                r.slot, r.admitted = slot, now()
                active[slot] = r
                queue.popleft()
            max_active = max(max_active, len(active))
            if not active:
                if queue:
                    raise RuntimeError(f"request {queue[0].rid} does not fit an empty batch")
                if i < len(reqs) and realtime:
                    sleep(max(0.0, reqs[i].arrival - now()))
                continue
            self.batch.step(self.chunk)
            chunks += 1
            left = self.batch.poll()
            for slot, r in list(active.items()):
                if left[slot] == 0:
                    res = self.batch.state(slot)
                    r.done = now()
                    if self.keep_results:
                        r.result = res
                    self.batch.remove(slot)
                    del active[slot]
                    steps_done += r.nsteps * r.prob.interior
        wall = now()
        lat = np.array([r.latency for r in reqs])
        return {"requests": len(reqs), "wall_s": wall, "chunks": chunks, "max_active": max_active,
                "cell_updates": steps_done, "cell_updates_per_s": steps_done / wall if wall > 0 else 0.0,
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "mean_s": float(lat.mean()) if len(lat) else None}


def atmosphere_request_maker(sizes=((128, 256), (256, 512), (384, 768), (512, 1024)),
                             period=(120.0, 600.0), amp=(50.0, 500.0), steps=(200, 2000)):
    """Requests of driven stratified-atmosphere x-z slices: (nx, nz) drawn from
    `sizes`, driver period U[period], amplitude U[amp], run length U[steps]."""
    from . import problems

    def make(i, rng):
        nx, nz = sizes[rng.integers(len(sizes))]
        prob = problems.atmosphere(nz, nx)
        prob.driver["period"] = float(rng.uniform(*period))
        prob.driver["amp"] = float(rng.uniform(*amp))
        return prob, int(rng.integers(steps[0], steps[1] + 1))

    return make


__all__ = ["Request", "Server", "poisson_stream", "atmosphere_request_maker", "PREC_MIXED"]
