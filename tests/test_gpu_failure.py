"""Failure detection without a GPU fault: a simulation whose state holds a
NaN (made on the host) drives its wave speeds and dt non-finite.  The dt and
finish logic then set the simulation's device status, so that

* a single-simulation context reports SMAUG_ERR_NONFINITE from smaug_sync;
* in a batch, smaug_batch_sync reports SMAUG_ERR_NONFINITE and names the slot,
  the failed simulation stops taking steps, and every other simulation runs
  on and finishes with the same bits it gives alone.
"""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_FP64, PREC_MIXED, Batch, Engine, SmaugError, footprint, problems

pytestmark = pytest.mark.gpu

SMAUG_ERR_NONFINITE = -4


def _poisoned(prob):
    w = np.array(prob.w, copy=True)
    w[0, prob.n[1] // 2, prob.n[0] // 2] = np.nan  # density at an inner cell
    return w


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_context_reports_nonfinite(need_gpu, prec):
    prob = problems.orszag_tang(32)
    e = Engine(prob, rk4=True, precision=prec)
    e.set_state(_poisoned(prob))
    e.step(3)
    with pytest.raises(SmaugError) as ex:
        e.sync()
    assert f"({SMAUG_ERR_NONFINITE})" in str(ex.value)
    # a clean state loads and steps again in the same context
    e.set_state(prob.w)
    e.step(2)
    e.sync()
    e.close()


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_batch_names_failed_slot_others_unaffected(need_gpu, prec):
    probs = [problems.orszag_tang(n, rho_noise=0.01, seed=s) for n, s in ((32, 1), (40, 2), (24, 3))]
    nsteps = 12
    fp = sum(footprint(p, prec) for p in probs)
    b = Batch(2, precision=prec, arena_bytes=fp + (1 << 20), max_sims=4)
    slots = [b.add(p, nsteps, w=(_poisoned(p) if i == 1 else None)) for i, p in enumerate(probs)]
    b.step(nsteps)
    rc, bad, msg = b.status()
    assert rc == SMAUG_ERR_NONFINITE
    assert bad == slots[1] and f"simulation {slots[1]}" in msg
    left = b.poll()
    assert left[slots[0]] == 0 and left[slots[2]] == 0
    assert left[slots[1]] > 0  # stopped on the device
    for i in (0, 2):
        e = Engine(probs[i], rk4=True, precision=prec)
        e.step(nsteps)
        assert np.array_equal(b.state(slots[i]), e.state()), i
        e.close()
    b.close()
