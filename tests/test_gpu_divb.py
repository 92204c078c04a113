"""Divergence-of-B source terms on the GPU (needs a GPU).

The reference's cudivb (divb.cu:165-336, divbon = divbfix = 1), 2-D, against
the oracle, which matches the reference's own divb.cu bit for bit
(tests/test_oracle.py): the FMA-free build bit for bit, the production FP64
build within 1e-6 and the mixed path within 1e-5 relative L2 per field.
"""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_MIXED, Engine, SmaugError, problems

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def noisy_ot(n, btype=None):
    """Orszag-Tang with B noise (its initial field is divergence-free)."""
    prob = problems.orszag_tang(n)
    rng = np.random.default_rng(5)
    for k in range(2):
        prob.w[4 + k] += 0.02 * rng.standard_normal(prob.w.shape[1:])
    if btype:
        prob.btype = tuple(btype)
    prob.divb = 1
    return prob


def rel_l2(a, b):
    out = []
    sl = (slice(None),) + tuple(slice(2, -2) for _ in range(a.ndim - 1))
    a, b = a[sl], b[sl]
    for f in range(a.shape[0]):
        nb = np.linalg.norm(b[f])
        out.append(np.linalg.norm(a[f] - b[f]) / (nb if nb > 0 else 1.0))
    return np.array(out)


@pytest.mark.parametrize("btype,rk4,steps", [(None, True, 6), (None, False, 8), ((4, 5), True, 5)])
def test_exact_build_bit_exact_vs_oracle(need_gpu, btype, rk4, steps):
    prob = noisy_ot(36, btype)
    o = Oracle(prob)
    eng = Engine(prob, rk4=rk4, exact=True)
    for s in range(steps):
        o.step(1, rk4=rk4)
        eng.step(1)
        assert eng.scalars()["dt"] == o.dt, (s, eng.scalars()["dt"], o.dt)
    w = eng.state()
    assert np.array_equal(w, o.w), rel_l2(w, o.w)


@pytest.mark.parametrize("precision,rk4,tol", [(0, True, 1e-6), (0, False, 1e-6), (PREC_MIXED, True, 1e-5)])
def test_fast_paths_within_tolerance(need_gpu, precision, rk4, tol):
    prob = noisy_ot(40)
    o = Oracle(prob)
    o.step(6, rk4=rk4)
    eng = Engine(prob, rk4=rk4, precision=precision)
    eng.step(6)
    err = rel_l2(eng.state(), o.w)
    assert np.all(err < tol), err
    # and the terms act
    prob.divb = 0
    off = Oracle(prob)
    off.step(6, rk4=rk4)
    assert rel_l2(off.w, o.w).max() > 100 * tol


def test_divb_is_rejected_in_3d(need_gpu):
    prob = problems.blast_wave(12)
    prob.divb = 1
    with pytest.raises(SmaugError):
        Engine(prob, rk4=True)
