"""Metric checks at admission (needs a GPU): smaug_batch_add takes the
reference's per-cell metric arrays, keeps one line per dimension and the last
dimension's full array, and rejects a metric that is not a tensor-product grid
on the inner cells or has a non-positive entry (the ghost layers of the
reference's own metric differ from the lines in the last bits, and pass)."""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_MIXED, SmaugError, problems
from smaug_b200.batch import Batch

pytestmark = pytest.mark.gpu


def metric(prob):
    return np.concatenate([a.ravel() for a in prob.delx()])


@pytest.mark.parametrize("kind", ["ot", "blast"])
def test_explicit_metric_gives_the_default_bits(need_gpu, kind):
    prob = problems.orszag_tang(40) if kind == "ot" else problems.blast_wave(12, seed=2)
    D = prob.ndim
    out = []
    for explicit in (False, True):
        b = Batch(D, precision=PREC_MIXED, arena_bytes=128 << 20, max_sims=1)
        s = b.add(prob, 3, delx=metric(prob) if explicit else None)
        b.step(3)
        out.append((b.state(s), b.scalars(s)))
        b.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


@pytest.mark.parametrize("kind", ["ot", "blast"])
@pytest.mark.parametrize("defect", ["inner", "nonpositive_ghost", "size"])
def test_bad_metric_is_rejected_and_frees_nothing(need_gpu, kind, defect):
    prob = problems.orszag_tang(24) if kind == "ot" else problems.blast_wave(10, seed=2)
    D = prob.ndim
    m = [a.copy() for a in prob.delx()]
    if defect == "inner":       # one inner cell off its line, in the last dimension
        m[D - 1][(3,) * D] *= 1.0 + 1e-12
    elif defect == "nonpositive_ghost":
        m[0][(0,) * D] = 0.0
    flat = np.concatenate([a.ravel() for a in m])
    if defect == "size":
        flat = flat[:-1]
    b = Batch(D, precision=PREC_MIXED, arena_bytes=64 << 20, max_sims=2)
    with pytest.raises(SmaugError):
        b.add(prob, 2, delx=flat)
    # the slot and its memory are still free: a good simulation is admitted
    # and steps
    s = b.add(prob, 2)
    assert s is not None
    b.step(2)
    assert np.isfinite(b.state(s)).all()
    b.close()


@pytest.mark.parametrize("kind", ["ot", "blast"])
@pytest.mark.parametrize("defect", ["inner", "nonpositive_ghost", "count"])
def test_set_metric_rejects_a_bad_metric(need_gpu, kind, defect):
    """smaug_set_metric checks the metric on the host, in one pass in storage
    order: SMAUG_ERR_ARG, and the context keeps its metric and still steps
    to the same bits as a context that never saw the bad one."""
    import ctypes

    from smaug_b200 import Engine
    prob = problems.orszag_tang(24) if kind == "ot" else problems.blast_wave(10, seed=2)
    D = prob.ndim
    m = [a.copy() for a in prob.delx()]
    if defect == "inner":
        m[D - 1][(3,) * D] *= 1.0 + 1e-12
    elif defect == "nonpositive_ghost":
        m[0][(0,) * D] = -1.0
    flat = np.ascontiguousarray(np.concatenate([a.ravel() for a in m]))
    count = flat.size - (1 if defect == "count" else 0)
    e = Engine(prob, rk4=True, precision=PREC_MIXED)
    rc = e.lib.smaug_set_metric(e.h, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), count)
    assert rc != 0
    e.step(2)
    ref = Engine(prob, rk4=True, precision=PREC_MIXED)
    ref.step(2)
    assert np.array_equal(e.state(), ref.state())
    e.close()
    ref.close()
