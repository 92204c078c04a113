"""Batches of simulations of uneven sizes (needs a GPU).

Bar: a simulation's results in a batch are bit-identical to those of a
single-simulation context with the same parameters -- the same tile body does
the same arithmetic per cell, and the wave-speed and viscosity maxima are
order-independent -- whatever else is in the batch, whatever the tile shape,
and however many steps the others take.
"""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_FP64, PREC_MIXED, Batch, Engine, footprint, problems

pytestmark = pytest.mark.gpu


def ot_mix():
    return [problems.orszag_tang(24), problems.orszag_tang(40, b0_scale=1.3, rho_noise=0.01, seed=7),
            problems.orszag_tang(33, b0_scale=0.7, rho_noise=0.01, seed=8), problems.orszag_tang(17)]


def alone(prob, steps, precision, **kw):
    e = Engine(prob, rk4=True, precision=precision, **kw)
    e.step(steps)
    w, s = e.state(), e.scalars()
    e.close()
    return w, s


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_batch_matches_single_simulation(need_gpu, precision):
    probs = ot_mix()
    steps = [6, 3, 9, 5]
    b = Batch(2, precision=precision, arena_bytes=256 << 20, max_sims=8)
    slots = [b.add(p, k) for p, k in zip(probs, steps)]
    b.step(12)  # more than any simulation asks for: finished ones stop
    b.sync()
    left = b.poll()
    assert all(left[s] == 0 for s in slots)
    for p, k, s in zip(probs, steps, slots):
        w_ref, sc_ref = alone(p, k, precision)
        assert np.array_equal(b.state(s), w_ref), (p.n, k)
        sc = b.scalars(s)
        assert sc["dt"] == sc_ref["dt"] and sc["steps"] == k
        assert sc["maxviscoef"] == sc_ref["maxviscoef"]


def test_batch_tile_shapes_and_graph_replay_are_identical(need_gpu):
    probs = ot_mix()[:3]
    ref = [alone(p, 21, PREC_MIXED)[0] for p in probs]
    for v in range(11):
        b = Batch(2, precision=PREC_MIXED, arena_bytes=256 << 20, max_sims=4)
        slots = [b.add(p, 21) for p in probs]
        b.set_variant(v)
        b.step(21)  # one 16-step graph replay and five 1-step replays
        for s, r in zip(slots, ref):
            assert np.array_equal(b.state(s), r), v
        b.close()


def test_batch_3d(need_gpu):
    probs = [problems.blast_wave(12, seed=3), problems.blast_wave(16, seed=4), problems.blast_wave(10, seed=5)]
    b = Batch(3, precision=PREC_MIXED, arena_bytes=256 << 20, max_sims=4)
    slots = [b.add(p, 4) for p in probs]
    v, ms = b.tune(reps=2)
    assert 0 <= v < 10 and len(ms) == 10 and all(m > 0 for m in ms)
    b.step(4)
    for p, s in zip(probs, slots):
        assert np.array_equal(b.state(s), alone(p, 4, PREC_MIXED)[0])


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_batch_3d_tile_shapes_are_identical(need_gpu, precision):
    """Every 3-D tile shape (256- and 512-thread tiles, 1 to 4 blocks per SM,
    ragged grids) gives the bits of the simulation run alone."""
    probs = [problems.blast_wave(12, seed=3), problems.blast_wave(10, seed=5)]
    ref = [alone(p, 4, precision)[0] for p in probs]
    for v in range(10):
        b = Batch(3, precision=precision, arena_bytes=256 << 20, max_sims=4)
        slots = [b.add(p, 4) for p in probs]
        b.set_variant(v)
        b.step(4)
        for s, r in zip(slots, ref):
            assert np.array_equal(b.state(s), r), v
        b.close()


def test_batch_admission_by_footprint(need_gpu):
    small, big = problems.orszag_tang(24), problems.orszag_tang(64)
    fs, fb = footprint(small, PREC_MIXED), footprint(big, PREC_MIXED)
    b = Batch(2, precision=PREC_MIXED, arena_bytes=fb + fs + 4096, max_sims=4)
    s_big = b.add(big, 5)
    s_small = b.add(small, 5)
    assert s_big is not None and s_small is not None
    assert b.add(big, 5) is None  # no room
    b.step(2)
    b.remove(s_big)
    assert b.info()["sims"] == 1
    s2 = b.add(big, 3)  # the freed block is reused while the small one runs on
    assert s2 is not None
    b.step(5)
    assert np.array_equal(b.state(s_small), alone(small, 5, PREC_MIXED)[0])
    assert np.array_equal(b.state(s2), alone(big, 3, PREC_MIXED)[0])


def test_batch_fixed_dt_and_dt_rule_mixed(need_gpu):
    p1, p2 = problems.orszag_tang(20), problems.orszag_tang(28)
    b = Batch(2, precision=PREC_FP64, arena_bytes=64 << 20, max_sims=2)
    s1 = b.add(p1, 4, dt_mode=0, dt0=1e-3)
    s2 = b.add(p2, 4)
    b.step(4)
    assert np.array_equal(b.state(s1), alone(p1, 4, PREC_FP64, dt_mode=0, dt0=1e-3)[0])
    assert np.array_equal(b.state(s2), alone(p2, 4, PREC_FP64)[0])
    assert b.scalars(s1)["dt"] == 1e-3


def test_batch_atmosphere_slices_with_driver(need_gpu):
    """Driven atmosphere slices of different sizes and driver periods in one
    batch give the bits they give alone (the driver clock is per simulation)."""
    probs = [problems.atmosphere(40, 20, noise=1e-3, seed=1), problems.atmosphere(64, 32, noise=1e-3, seed=2),
             problems.atmosphere(48, 16, noise=1e-3, seed=3)]
    for k, p in enumerate(probs):
        p.driver["amp"] = 1.0e3 * (k + 1)
        p.driver["period"] = 2.0 + k
    steps = [5, 7, 3]
    b = Batch(2, precision=PREC_MIXED, arena_bytes=128 << 20, max_sims=4)
    slots = [b.add(p, k) for p, k in zip(probs, steps)]
    b.step(8)
    for p, k, s in zip(probs, steps, slots):
        assert np.array_equal(b.state(s), alone(p, k, PREC_MIXED)[0])
