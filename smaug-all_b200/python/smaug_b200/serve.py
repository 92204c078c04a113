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
    methods add / step / poll_begin / poll_end / state_async / io_wait /
    remove).

    The device is never left without queued work while any simulation is
    active: the loop keeps `depth` chunks of `chunk` steps queued, each
    followed by a snapshot of the steps left (poll_begin).  It then waits for
    the oldest snapshot only -- the chunks queued behind it keep the GPU busy
    -- retires the simulations that had finished by it (their states are read
    on the batch's read-back stream after that snapshot, into pinned buffers,
    while later chunks run), and admits waiting requests as slots and memory
    free up (admissions run on their own stream and do not wait for the
    queued chunks either)."""

    def __init__(self, batch, chunk: int = 8, keep_results: bool = True, depth: int = 2, time_chunks: bool = False):
        self.batch = batch
        self.chunk = chunk
        self.keep_results = keep_results
        self.depth = max(1, depth)
        # CUDA events around every chunk on the batch's stream: the device's
        # busy time while serving (needs torch and a batch with a stream)
        self.time_chunks = time_chunks
        self._pool: dict = {}

    def _chunk_events(self):
        import torch
        st = torch.cuda.ExternalStream(self.batch.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        return st, e0, e1

    def _buffer(self, shape):
        free = self._pool.setdefault(shape, [])
        if free:
            return free.pop()
        try:
            import torch
            if torch.cuda.is_available():
                return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        except Exception:
            pass
        return np.empty(shape, dtype=np.float64)

    def run(self, requests, realtime: bool = True, clock=time.perf_counter, sleep=time.sleep,
            stop_after: float | None = None) -> dict:
        """Serve `requests` (arrival times in seconds from the start).  With
        stop_after, no request is admitted and no chunk is queued after that
        many seconds; the loop then ends once the queued chunks are done, and
        the statistics cover the requests completed by then (cell_updates
        counts every step executed, of unfinished simulations too)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        queue: deque = deque()
        active: dict = {}     # slot -> request
        steps_seen: dict = {}  # rid -> steps executed as of the last snapshot
        inflight: deque = deque()  # (ticket, [(slot, rid)]) in queue order
        i, chunks, max_active = 0, 0, 0
        samples = []  # (t, waiting, active)
        events = []   # (start, end) of every chunk on the device
        stopped = False
        while True:
            t = now()
            if stop_after is not None and t >= stop_after:
                stopped = True
            while not stopped and i < len(reqs) and (reqs[i].arrival <= t or not realtime):
                queue.append(reqs[i])
                i += 1
            while queue and not stopped:  # first come first served: the head waits until it fits
                r = queue[0]
                slot = self.batch.add(r.prob, r.nsteps)
                if slot is None:
                    break
                r.slot, r.admitted = slot, now()
                active[slot] = r
                steps_seen[r.rid] = 0
                queue.popleft()
            max_active = max(max_active, len(active))
            samples.append((round(t, 3), len(queue), len(active)))
            if active and not stopped and len(inflight) < self.depth:
                if self.time_chunks:
                    st_, e0, e1 = self._chunk_events()
                    e0.record(st_)
                self.batch.step(self.chunk)
                if self.time_chunks:
                    e1.record(st_)
                    events.append((e0, e1))
                chunks += 1
                inflight.append((self.batch.poll_begin(), [(s_, r_.rid) for s_, r_ in active.items()]))
                if len(inflight) < self.depth:
                    continue  # fill the pipeline first
            if inflight:
                ticket, snap = inflight.popleft()
                left = self.batch.poll_end(ticket)
                done = []
                for slot, rid in snap:
                    r = active.get(slot)
                    if r is None or r.rid != rid:
                        continue
                    steps_seen[rid] = r.nsteps - int(left[slot])
                    if left[slot] == 0:
                        buf = self._buffer(r.prob.w.shape)
                        self.batch.state_async(slot, buf)
                        self.batch.remove(slot)
                        del active[slot]
                        done.append((r, buf))
                if done:
                    self.batch.io_wait()
                    td = now()
                    for r, buf in done:
                        r.done = td
                        if self.keep_results:
                            r.result = buf.copy()
                        self._pool[r.prob.w.shape].append(buf)
                continue
            if stopped or (i >= len(reqs) and not queue and not active):
                break
            if not active:
                if queue:
                    raise RuntimeError(f"request {queue[0].rid} does not fit an empty batch")
                if i < len(reqs) and realtime:
                    sleep(max(0.0, reqs[i].arrival - now()))
        wall = now()
        fin = [r for r in reqs if r.done is not None]
        lat = np.array([r.latency for r in fin])
        cell_updates = sum(steps_seen.get(r.rid, 0) * r.prob.interior for r in reqs)
        self.latencies = [float(x) for x in lat]
        dev = {}
        if events:
            events[-1][1].synchronize()
            busy = sum(a.elapsed_time(b) for a, b in events) / 1e3
            span = events[0][0].elapsed_time(events[-1][1]) / 1e3
            dev = {"gpu_busy_s": busy, "gpu_span_s": span, "gpu_busy_fraction": busy / span if span > 0 else 0.0}
        return {**dev, "requests": len(reqs), "completed": len(fin), "unfinished_active": len(active),
                "still_waiting": len(queue) + (len(reqs) - i), "wall_s": wall, "chunks": chunks,
                "max_active": max_active, "cell_updates": cell_updates,
                "cell_updates_per_s": cell_updates / wall if wall > 0 else 0.0,
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "mean_s": float(lat.mean()) if len(lat) else None,
                "queue_samples": samples[:: max(1, len(samples) // 200)]}


def shard(requests, rank: int, world: int) -> list:
    """The requests one of `world` replicas serves: every world-th request in
    arrival order, starting at `rank` (each replica runs its own batch on its
    own GPU; no data passes between them)."""
    ordered = sorted(requests, key=lambda r: r.arrival)
    return [r for k, r in enumerate(ordered) if k % world == rank]


def merge_stats(per_rank: list) -> dict:
    """Whole-stream statistics from the replicas' (stats, latencies) pairs:
    requests and cell-updates add up, the wall time is the slowest
    replica's, the percentiles are over every completed request."""
    lat = np.concatenate([np.asarray(l, dtype=float) for _, l in per_rank]) if per_rank else np.zeros(0)
    wall = max(st["wall_s"] for st, _ in per_rank)
    cu = sum(st["cell_updates"] for st, _ in per_rank)
    return {"replicas": len(per_rank), "requests": sum(st["requests"] for st, _ in per_rank),
            "completed": int(len(lat)), "wall_s": wall, "cell_updates": cu,
            "cell_updates_per_s": cu / wall if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None}


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


__all__ = ["Request", "Server", "poisson_stream", "atmosphere_request_maker", "shard", "merge_stats", "PREC_MIXED"]
