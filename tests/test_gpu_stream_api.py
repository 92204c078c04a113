"""Stage- and stream-level entry points of the C ABI (needs a GPU):
smaug_stage runs one Runge-Kutta stage of the current step on the caller's
stream, smaug_step_on runs whole steps there.  Stages 1..4 of a step, or
steps on another stream, give the same bits as smaug_step on the context's
own stream; stages out of order are refused."""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_FP64, PREC_MIXED, Engine, SmaugError, problems

pytestmark = pytest.mark.gpu

MODES = [  # (rk4, exact, precision)
    (True, False, PREC_FP64),
    (True, False, PREC_MIXED),
    (True, True, PREC_FP64),
    (False, True, PREC_FP64),
    (False, False, PREC_FP64),
]


@pytest.mark.parametrize("rk4,exact,prec", MODES)
def test_stages_equal_steps(need_gpu, rk4, exact, prec):
    import torch
    prob = problems.orszag_tang(40, rho_noise=0.01, seed=3)
    a = Engine(prob, rk4=rk4, exact=exact, precision=prec)
    b = Engine(prob, rk4=rk4, exact=exact, precision=prec)
    s = torch.cuda.Stream()
    nst = 4 if rk4 else 1
    for _ in range(5):
        a.step(1)
        for k in range(1, nst + 1):
            b.stage(k, s.cuda_stream)
    s.synchronize()
    assert np.array_equal(a.state(), b.state())
    sa, sb = a.scalars(), b.scalars()
    assert sa["dt"] == sb["dt"] and sa["steps"] == sb["steps"] == 5


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_step_on_caller_stream(need_gpu, prec):
    import torch
    prob = problems.blast_wave(16, seed=4)
    a = Engine(prob, rk4=True, precision=prec)
    b = Engine(prob, rk4=True, precision=prec)
    s = torch.cuda.Stream()
    a.step(19)  # 16-step graph + 3 single-step graphs
    b.step_on(19, s.cuda_stream)
    # context work queued after the caller-stream steps waits for them
    assert np.array_equal(a.state(), b.state())


def test_stage_order_is_enforced(need_gpu):
    prob = problems.orszag_tang(24)
    e = Engine(prob, rk4=True)
    with pytest.raises(SmaugError):
        e.stage(2)
    e.stage(1)
    with pytest.raises(SmaugError):
        e.step(1)  # a step begun stage by stage is unfinished
    with pytest.raises(SmaugError):
        e.stage(3)
    for k in (2, 3, 4):
        e.stage(k)
    e.step(1)
    e.sync()
