"""The end-to-end pipeline of bench.py against a fake batch (CPU).

The fake keeps each simulation's step budget, takes poll snapshots behind
the steps queued so far, and accepts a read only for a simulation that had
finished in the last snapshot waited for -- the contract of
smaug_batch_poll_begin / poll_end / get_state_async.  Every simulation must
take exactly its steps and be read back once, whatever the ensemble size and
step count.
"""
from __future__ import annotations

import numpy as np
import pytest

import bench


class FakeBatch:
    def __init__(self):
        self.left, self.taken, self.snaps, self.nt = {}, {}, {}, 0
        self.seen, self.queued_reads, self.reads = None, [], []

    def add(self, prob, steps, w=None, delx=None):
        slot = len(self.left)
        self.left[slot], self.taken[slot] = steps, 0
        return slot

    def step(self, n):
        for _ in range(n):
            for k in self.left:
                if self.left[k] > 0:
                    self.left[k] -= 1
                    self.taken[k] += 1

    def poll_begin(self):
        assert len(self.snaps) < 4, "at most 4 snapshots wait at a time"
        self.nt += 1
        self.snaps[self.nt] = np.array([self.left[k] for k in sorted(self.left)])
        return self.nt

    def poll_end(self, ticket):
        self.seen = self.snaps.pop(ticket)
        return self.seen

    def state_async(self, slot, out):
        assert self.seen is not None and self.seen[slot] == 0, "read of a simulation not finished in the snapshot"
        self.queued_reads.append((slot, out))

    def io_wait(self):
        for slot, out in self.queued_reads:
            out[...] = slot
            self.reads.append(slot)
        self.queued_reads = []


@pytest.mark.parametrize("n,steps", [(96, 20), (96, 2), (96, 1), (5, 20), (17, 13), (8, 3)])
def test_e2e_pipeline_steps_and_reads(n, steps):
    b = FakeBatch()
    outs = [np.full(4, -1.0) for _ in range(n)]
    slots = bench.e2e_pipeline(b, list(range(n)), [None] * n, [None] * n, outs, steps)
    assert slots == list(range(n))
    assert all(b.taken[k] == steps for k in b.taken)
    assert sorted(b.reads) == list(range(n))
    assert all(np.all(o == k) for k, o in enumerate(outs))
    # the first members are read before the last steps are queued when the
    # admissions queued steps of their own
    if n >= 2 * bench.E2E_STEP_EVERY and steps > 2:
        assert b.reads[0] == 0
