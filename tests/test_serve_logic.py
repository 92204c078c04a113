"""Host logic of the serving loop (no GPU): admission by footprint, first
come first served, chunked stepping, retirement, latency accounting.  A fake
batch stands in for the device batch."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from smaug_b200.serve import Request, Server, poisson_stream


class FakeBatch:
    def __init__(self, capacity, max_sims=8):
        self.capacity, self.used = capacity, 0
        self.left = np.full(max_sims, -1, dtype=np.int64)
        self.size = {}
        self.log = []

    def add(self, prob, nsteps):
        need = prob.interior
        free = [s for s in range(len(self.left)) if self.left[s] < 0]
        if not free or self.used + need > self.capacity:
            return None
        s = free[0]
        self.left[s] = nsteps
        self.size[s] = need
        self.used += need
        self.log.append(("add", prob.tag, s))
        return s

    def step(self, n):
        act = self.left > 0
        self.left[act] = np.maximum(self.left[act] - n, 0)

    def poll(self):
        return self.left.copy()

    # the asynchronous protocol: a snapshot per ticket, reads filled at io_wait
    def poll_begin(self):
        self.snaps = getattr(self, "snaps", [])
        self.snaps.append(self.left.copy())
        self.log.append(("poll_begin", len(self.snaps) - 1))
        return len(self.snaps) - 1

    def poll_end(self, ticket):
        self.log.append(("poll_end", ticket))
        return self.snaps[ticket]

    def state_async(self, slot, out):
        out[...] = slot
        return out

    def io_wait(self):
        pass

    def state(self, slot):
        return np.full(3, slot, dtype=float)

    def remove(self, slot):
        self.used -= self.size.pop(slot)
        self.left[slot] = -1
        self.log.append(("remove", slot))


def prob(tag, cells):
    return SimpleNamespace(tag=tag, interior=cells, w=np.zeros(3))


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3  # every clock read advances simulated time a little
        return self.t

    def sleep(self, dt):
        self.t += dt


def test_fifo_admission_and_retirement():
    reqs = [Request(0, prob("a", 6), 10, 0.0), Request(1, prob("b", 6), 3, 0.0), Request(2, prob("c", 2), 4, 0.0)]
    fb = FakeBatch(capacity=10)
    ck = Clock()
    st = Server(fb, chunk=2).run(reqs, realtime=True, clock=ck, sleep=ck.sleep)
    # b waits for a (head of line), c waits behind b although it would fit
    adds = [e for e in fb.log if e[0] == "add"]
    assert [a[1] for a in adds] == ["a", "b", "c"]
    first_remove = fb.log.index(("remove", 0))
    assert fb.log.index(("add", "b", 0)) > first_remove
    assert all(r.done is not None and r.latency > 0 for r in reqs)
    assert st["requests"] == 3 and st["cell_updates"] == 6 * 10 + 6 * 3 + 2 * 4
    assert st["p99_s"] >= st["p50_s"] > 0
    assert fb.used == 0


def test_idle_server_waits_for_arrivals():
    reqs = [Request(0, prob("a", 4), 2, 0.5), Request(1, prob("b", 4), 2, 2.0)]
    ck = Clock()
    st = Server(FakeBatch(100), chunk=4).run(reqs, clock=ck, sleep=ck.sleep)
    assert reqs[0].admitted >= 0.5 and reqs[1].admitted >= 2.0
    assert st["max_active"] == 1


def test_request_larger_than_the_arena_is_an_error():
    import pytest
    ck = Clock()
    with pytest.raises(RuntimeError):
        Server(FakeBatch(5)).run([Request(0, prob("big", 6), 1, 0.0)], clock=ck, sleep=ck.sleep)


def test_poisson_stream_is_seeded_and_ordered():
    mk = lambda i, rng: (prob(i, 1), int(rng.integers(1, 5)))  # noqa: E731
    a = poisson_stream(50, 40.0, mk, seed=777)
    b = poisson_stream(50, 40.0, mk, seed=777)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert np.all(gaps > 0) and 0.01 < gaps.mean() < 0.05
    assert len(poisson_stream(1000, 40.0, mk, duration=1.0)) < 80


def test_next_chunk_is_queued_before_the_last_is_waited_for():
    """With depth 2 the loop queues chunk k+1 (and its snapshot) before it
    waits for snapshot k: the device always has a chunk to run while the host
    retires and admits."""
    reqs = [Request(0, prob("a", 4), 6, 0.0), Request(1, prob("b", 4), 20, 0.0)]
    fb = FakeBatch(capacity=100)
    ck = Clock()
    Server(fb, chunk=2, depth=2).run(reqs, clock=ck, sleep=ck.sleep)
    ev = [e for e in fb.log if e[0] in ("poll_begin", "poll_end")]
    for k in range(len(fb.snaps) - 1):
        assert ev.index(("poll_begin", k + 1)) < ev.index(("poll_end", k)), k
    # a, done after 3 chunks, is retired from snapshot 2 while chunk 4 is queued
    assert fb.log.index(("remove", 0)) > fb.log.index(("poll_begin", 3))


def test_stop_after_reports_executed_work():
    reqs = [Request(i, prob(i, 3), 50, 0.01 * i) for i in range(6)]
    fb = FakeBatch(capacity=6)  # two at a time
    ck = Clock()
    st = Server(fb, chunk=5, depth=2).run(reqs, clock=ck, sleep=ck.sleep, stop_after=0.05)
    assert st["completed"] < 6 and st["completed"] + st["unfinished_active"] + st["still_waiting"] == 6
    done_work = sum(r.nsteps * 3 for r in reqs if r.done is not None)
    assert st["cell_updates"] >= done_work
