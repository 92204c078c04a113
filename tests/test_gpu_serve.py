"""Serving loop on the GPU: requests that arrive while others run are
admitted as memory frees up, their work overlaps on the device, and each
result is the same alone and in the mix (bit for bit: per-simulation dt,
driver clock and step budget, and the same stage kernel arithmetic)."""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_MIXED, Batch, Engine, footprint
from smaug_b200.serve import Server, atmosphere_request_maker, poisson_stream

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone(need_gpu):
    make = atmosphere_request_maker(sizes=((32, 48), (40, 64), (24, 40)), period=(2.0, 6.0), amp=(500.0, 2000.0),
                                    steps=(5, 20))
    reqs = poisson_stream(8, 200.0, make, seed=777)
    fp = [footprint(r.prob, PREC_MIXED) for r in reqs]
    # room for about three at a time: later arrivals queue and are admitted
    # as earlier ones finish
    b = Batch(2, precision=PREC_MIXED, arena_bytes=3 * max(fp) + 4096, max_sims=8)
    st = Server(b, chunk=4).run(reqs)
    assert st["requests"] == 8 and 1 < st["max_active"] <= 3
    for r in reqs:
        e = Engine(r.prob, rk4=True, precision=PREC_MIXED)
        e.step(r.nsteps)
        assert np.array_equal(r.result, e.state()), r.rid
        e.close()
    assert st["p99_s"] >= st["p50_s"] > 0
