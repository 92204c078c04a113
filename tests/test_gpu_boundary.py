"""Boundary types beyond periodic / contcd4 on the GPU (needs a GPU).

cont, fixed, symm and asymm (with per-field asymm masks on symm directions)
against the oracle, whose ghost fill matches the reference's own boundary
helpers bit for bit (tests/test_oracle.py).  Bar as in test_gpu_parity: the
FMA-free build bit for bit, the production FP64 build within 1e-6 and the
mixed path within 1e-5 relative L2 per field; a batch of simulations with
different boundaries gives each one's single-simulation bits.
"""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_MIXED, Engine, problems
from smaug_b200.batch import Batch

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FAST_RTOL = 1e-6
MIXED_RTOL = 1e-5

# bmask bits: 2-D m_x 1, m_y 2, B_x 4, B_y 5; 3-D m 1-3, B 5-7
CASES = [
    ("ot", 40, (3, 3), None, True, 6),
    ("ot", 40, (5, 5), None, True, 6),
    ("ot", 40, (6, 6), (0b10010, 0b100100), True, 6),
    ("ot", 36, (7, 7), None, False, 6),
    ("ot", 36, (0, 5), None, True, 6),
    ("ot", 36, (5, 3), None, False, 6),
    ("ot", 36, (6, 0), None, True, 6),
    ("blast", 14, (3, 3, 0), None, True, 4),
    ("blast", 14, (5, 5, 5), None, True, 4),
    ("blast", 14, (6, 6, 6), (0b100010, 0b1000100, 0b10001000), True, 4),
    ("blast", 14, (0, 3, 5), None, False, 4),
    ("ot", 36, (4, 5), None, True, 5),
    ("blast", 14, (4, 6, 5), None, True, 4),
]


def make(kind, n, btype, bmask):
    """The state's ghost cells get noise, so that they match no fill rule:
    fixed ghosts, and the cells the fill takes from them, then differ from
    anything a wrong fill would write."""
    prob = problems.orszag_tang(n) if kind == "ot" else problems.blast_wave(n, seed=11)
    prob.btype = tuple(btype)
    if bmask:
        prob.bmask = tuple(bmask)
    D = prob.ndim
    ghost = np.zeros(prob.w.shape[1:], dtype=bool)
    for d in range(D):
        sl = [slice(None)] * D
        ax = D - 1 - d
        sl[ax] = np.r_[0, 1, prob.n[d] - 2, prob.n[d] - 1]
        ghost[tuple(sl)] = True
    rng = np.random.default_rng(21)
    for f in range(2 + 2 * D):
        prob.w[f][ghost] *= 1.0 + 0.01 * rng.standard_normal(int(ghost.sum()))
    return prob


def rel_l2(a, b):
    out = []
    sl = (slice(None),) + tuple(slice(2, -2) for _ in range(a.ndim - 1))
    a, b = a[sl], b[sl]
    for f in range(a.shape[0]):
        nb = np.linalg.norm(b[f])
        out.append(np.linalg.norm(a[f] - b[f]) / (nb if nb > 0 else 1.0))
    return np.array(out)


@pytest.mark.parametrize("kind,n,btype,bmask,rk4,steps", CASES)
def test_exact_build_bit_exact_vs_oracle(need_gpu, kind, n, btype, bmask, rk4, steps):
    prob = make(kind, n, btype, bmask)
    o = Oracle(prob)
    eng = Engine(prob, rk4=rk4, exact=True)
    for s in range(steps):
        o.step(1, rk4=rk4)
        eng.step(1)
        assert eng.scalars()["dt"] == o.dt, (s, eng.scalars()["dt"], o.dt)
    w = eng.state()
    assert np.array_equal(w, o.w), rel_l2(w, o.w)
    assert eng.scalars()["maxviscoef"] == o.s.maxviscoef


@pytest.mark.parametrize("kind,n,btype,bmask,rk4,steps", CASES)
def test_fast_build_within_tolerance(need_gpu, kind, n, btype, bmask, rk4, steps):
    prob = make(kind, n, btype, bmask)
    o = Oracle(prob)
    o.step(steps, rk4=rk4)
    eng = Engine(prob, rk4=rk4, exact=False)
    eng.step(steps)
    err = rel_l2(eng.state(), o.w)
    assert np.all(err < FAST_RTOL), err


@pytest.mark.parametrize("kind,n,btype,bmask,rk4,steps", [c for c in CASES if c[4]])
def test_mixed_within_tolerance(need_gpu, kind, n, btype, bmask, rk4, steps):
    """The blast wave runs at fixed dt: under the dt rule its hyperviscosity
    switch reads rounding noise in the flat background, which any change of
    rounding amplifies (the FP64 FMA build drifts the same way)."""
    prob = make(kind, n, btype, bmask)
    dt_mode, dt0 = (1, 0.0) if kind == "ot" else (0, 2e-4)
    o = Oracle(prob, dt_fixed=dt0)
    o.step(steps, rk4=True, dt_mode=dt_mode)
    eng = Engine(prob, rk4=True, precision=PREC_MIXED, dt_mode=dt_mode, dt0=dt0)
    eng.step(steps)
    err = rel_l2(eng.state(), o.w)
    assert np.all(err < MIXED_RTOL), err


@pytest.mark.parametrize("precision", [0, PREC_MIXED])
def test_fixed_ghosts_keep_their_loaded_values(need_gpu, precision):
    """FP64 bit for bit; mixed to the FP32 value + compensation split."""
    prob = make("ot", 32, (5, 5), None)
    w0 = prob.w.copy()
    eng = Engine(prob, rk4=True, precision=precision)
    eng.step(5)
    w = eng.state()
    nw = 6
    assert not np.array_equal(w[:nw, 2:-2, 2:-2], w0[:nw, 2:-2, 2:-2])
    for sl in ((slice(None), slice(0, 2)), (slice(None), slice(-2, None)),
               (slice(0, 2), slice(None)), (slice(-2, None), slice(None))):
        got, want = w[(slice(0, nw),) + sl], w0[(slice(0, nw),) + sl]
        if precision == 0:
            assert np.array_equal(got, want)
        else:
            assert np.allclose(got, want, rtol=1e-13, atol=0)


@pytest.mark.parametrize("precision", [0, PREC_MIXED])
def test_batch_of_mixed_boundaries_matches_single_simulations(need_gpu, precision):
    probs = [make("ot", 32, (3, 0), None), make("ot", 28, (5, 5), None),
             make("ot", 36, (6, 6), (0b10010, 0b100100)), make("ot", 24, (0, 7), None)]
    b = Batch(2, precision=precision, arena_bytes=256 << 20, max_sims=4)
    slots = [b.add(p, 5) for p in probs]
    b.step(5)
    for p, s in zip(probs, slots):
        e = Engine(p, rk4=True, precision=precision)
        e.step(5)
        assert np.array_equal(b.state(s), e.state())
        e.close()
    b.close()
