"""The production kernels against the oracle at the benchmark configurations'
full sizes (needs a GPU).

The tiled production stage kernel (batch_stage_kernel, the one every
throughput number comes from) is run on each configuration's own grid, in
FP64 and in mixed precision, under the reference's dt rule, and compared with
the FP64 CPU oracle after a few RK4 steps (the oracle's cost bounds the step
counts):

  C1  Orszag-Tang 256^2, periodic, 10 steps
  C2  blast wave 128^3, periodic, 3 steps
  C4  one 768^2 member of the batched ensemble (B0 factor, 1 % density
      noise), 5 steps, inside a batch with a 128^2 member
  C3  stratified atmosphere 256 (vertical) x 128 x 128 with the driver,
      gravity, contcd4 vertical boundaries, 2 steps

Error measure per evolved field f over the inner cells:
||x_f - y_f||_2 / ||y_f||_2, where y is the oracle's state.  A field whose
oracle norm is zero, or below 1e-9 of the largest field norm (a field that
only rounding and second-order coupling have moved off zero, e.g. the
horizontal momenta of the driven atmosphere after two steps), is measured by
its absolute L2 divided by the largest field norm instead.

Bars: FP64 1e-6 per field (FMA contraction against the FMA-free oracle; the
method amplifies last-bit differences through its viscous dt), mixed 1e-5 per
field, dt within 1e-9 (FP64) and 2e-4 (mixed; its
viscous limit divides by a hyperviscosity coefficient formed in FP32).
"""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_FP64, PREC_MIXED, Batch, Engine, footprint, problems

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FP64_TOL, MIXED_TOL = 1e-6, 1e-5
NEAR_ZERO = 1e-9


def field_errors(x, y):
    """Per-field error of x against the reference y (inner cells, evolved fields)."""
    nw = 2 + 2 * (x.ndim - 1)
    sl = (slice(0, nw),) + tuple(slice(2, -2) for _ in range(x.ndim - 1))
    x, y = x[sl], y[sl]
    norms = np.array([np.linalg.norm(y[f]) for f in range(nw)])
    big = norms.max()
    out = []
    for f in range(nw):
        d = np.linalg.norm(x[f] - y[f])
        out.append(d / norms[f] if norms[f] > NEAR_ZERO * big else d / big)
    return np.array(out)


def _configs():
    return {
        "C1_ot256": (lambda: problems.orszag_tang(256), 10),
        "C2_blast128": (lambda: problems.blast_wave(128, seed=1234), 3),
        "C3_atmos256x128x128": (lambda: problems.atmosphere(256, 128, 128), 2),
    }


_oracle_cache: dict = {}


def _oracle(name, make, steps):
    if name not in _oracle_cache:
        prob = make()
        o = Oracle(prob)
        o.step(steps, rk4=True)
        _oracle_cache.clear()  # one configuration's states at a time (the 3-D ones are large)
        _oracle_cache[name] = (prob, o.w.copy(), o.dt)
    return _oracle_cache[name]


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", list(_configs()))
def test_production_kernel_vs_oracle_at_config_size(need_gpu, name, prec):
    make, steps = _configs()[name]
    prob, w_ref, dt_ref = _oracle(name, make, steps)
    e = Engine(prob, rk4=True, precision=prec)
    e.step(steps)
    e.sync()
    err = field_errors(e.state(), w_ref)
    dt = e.scalars()["dt"]
    e.close()
    tol = FP64_TOL if prec == PREC_FP64 else MIXED_TOL
    assert np.all(err <= tol), (name, err)
    assert abs(dt - dt_ref) <= (1e-9 if prec == PREC_FP64 else 2e-4) * dt_ref, (dt, dt_ref)


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_ensemble_768_member_in_batch_vs_oracle(need_gpu, prec):
    """C4: the ensemble's first 768^2 member, with a 128^2 member beside it in
    one batch (one persistent launch per stage over both work lists)."""
    ens = problems.ensemble(96, seed=4242)
    big = next(p for p in ens if p.n[0] == 772)
    small = next(p for p in ens if p.n[0] == 132)
    steps = 5
    o = Oracle(big)
    o.step(steps, rk4=True)
    fp = footprint(big, prec) + footprint(small, prec)
    b = Batch(2, precision=prec, arena_bytes=fp + (1 << 20), max_sims=2)
    s_big = b.add(big, steps)
    b.add(small, steps)
    b.step(steps)
    b.sync()
    err = field_errors(b.state(s_big), o.w)
    dt = b.scalars(s_big)["dt"]
    b.close()
    tol = FP64_TOL if prec == PREC_FP64 else MIXED_TOL
    assert np.all(err <= tol), err
    assert abs(dt - o.dt) <= (1e-9 if prec == PREC_FP64 else 2e-4) * o.dt
