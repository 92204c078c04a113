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

Bars:
* FP64 under the dt rule: 1e-6 per field (FMA contraction against the
  FMA-free oracle; the method amplifies last-bit differences through its
  viscous dt), dt within 1e-9;
* mixed at a fixed dt (half the dt the rule reaches): 1e-5 per field, the
  north-star bar on the arithmetic itself;
* mixed under the dt rule: dt within 2e-3 of the oracle's, and 1e-4 per field
  -- a different dt moves the state by about that relative amount times the
  state's change over the run.  The viscous limit divides by the largest
  hyperviscosity coefficient, max|d3 q| / max|d1 q| with q formed from FP32
  states; the third differences shrink as (k dx)^3 with resolution, so FP32
  rounding of q weighs more on finer grids (8e-4 measured on the 256^2 vortex
  after 10 steps, against 2e-5 on 48^2).
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


MIXED_DT_RULE_TOL = 1e-4

_oracle_cache: dict = {}


def _oracle(name, make, steps, fixed: bool):
    """The oracle's state after `steps` RK4 steps under the dt rule, or at a
    fixed dt of half the rule's last dt (one configuration cached at a time:
    the 3-D states are large)."""
    key = (name, fixed)
    if key not in _oracle_cache:
        rule = [v for k, v in _oracle_cache.items() if k == (name, False)]
        if fixed and not rule:
            _oracle(name, make, steps, False)
            rule = [_oracle_cache[(name, False)]]
        for k in [k for k in _oracle_cache if k[0] != name]:
            del _oracle_cache[k]
        prob = rule[0][0] if rule else make()
        dt0 = 0.5 * rule[0][2] if fixed else 0.0
        o = Oracle(prob, dt_fixed=dt0)
        o.step(steps, rk4=True, dt_mode=0 if fixed else 1)
        _oracle_cache[key] = (prob, o.w.copy(), o.dt)
    return _oracle_cache[key]


@pytest.mark.parametrize("mode", ["fp64-dt_rule", "mixed-fixed_dt", "mixed-dt_rule"])
@pytest.mark.parametrize("name", list(_configs()))
def test_production_kernel_vs_oracle_at_config_size(need_gpu, name, mode):
    make, steps = _configs()[name]
    prec = PREC_FP64 if mode.startswith("fp64") else PREC_MIXED
    fixed = mode.endswith("fixed_dt")
    prob, w_ref, dt_ref = _oracle(name, make, steps, fixed)
    kw = {"dt_mode": 0, "dt0": dt_ref} if fixed else {}
    e = Engine(prob, rk4=True, precision=prec, **kw)
    e.step(steps)
    e.sync()
    err = field_errors(e.state(), w_ref)
    dt = e.scalars()["dt"]
    e.close()
    tol = FP64_TOL if prec == PREC_FP64 else (MIXED_TOL if fixed else MIXED_DT_RULE_TOL)
    assert np.all(err <= tol), (name, mode, err)
    assert abs(dt - dt_ref) <= (1e-9 if prec == PREC_FP64 else 2e-3) * dt_ref, (dt, dt_ref)


@pytest.mark.parametrize("mode", ["fp64-dt_rule", "mixed-fixed_dt"])
def test_ensemble_768_member_in_batch_vs_oracle(need_gpu, mode):
    """C4: the ensemble's first 768^2 member, with a 128^2 member beside it in
    one batch (one persistent launch per stage over both work lists)."""
    ens = problems.ensemble(96, seed=4242)
    big = next(p for p in ens if p.n[0] == 772)
    small = next(p for p in ens if p.n[0] == 132)
    steps = 5
    prec = PREC_FP64 if mode.startswith("fp64") else PREC_MIXED
    fixed = mode.endswith("fixed_dt")
    dt0 = 0.0
    if fixed:
        probe = Oracle(big)
        probe.step(1, rk4=True)
        dt0 = 0.5 * probe.dt
    o = Oracle(big, dt_fixed=dt0)
    o.step(steps, rk4=True, dt_mode=0 if fixed else 1)
    fp = footprint(big, prec) + footprint(small, prec)
    b = Batch(2, precision=prec, arena_bytes=fp + (1 << 20), max_sims=2)
    kw = {"dt_mode": 0, "dt0": dt0} if fixed else {}
    s_big = b.add(big, steps, **kw)
    b.add(small, steps, **kw)
    b.step(steps)
    b.sync()
    err = field_errors(b.state(s_big), o.w)
    dt = b.scalars(s_big)["dt"]
    b.close()
    tol = FP64_TOL if prec == PREC_FP64 else MIXED_TOL
    assert np.all(err <= tol), err
    assert abs(dt - o.dt) <= 1e-9 * o.dt
