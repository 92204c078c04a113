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
||x_f - y_f||_2 / ||y_f||_2, where y is the oracle's state; a field whose
oracle norm is zero, or below 1e-9 of the largest field norm (moved off zero
by rounding only), takes its absolute L2 over the largest field norm.

Bars:
* FP64 under the dt rule: 1e-6 per field (FMA contraction against the
  FMA-free oracle; the method amplifies last-bit differences through its
  viscous dt), every step's dt within 1e-9;
* mixed at a fixed dt (half the dt the rule reaches): per field
  max(1e-5, 4 x the FP32 storage floor).  The floor is the error of the FP64
  oracle whose evolved state is rounded to FP32 after every step and nothing
  else, at the same dt sequence: what storing the state in FP32 costs
  whatever the arithmetic.  The mixed path rounds each of the four stage
  inputs of a step (4 roundings per step against the floor's one), and was
  measured at 2.2-2.9 x the floor where the floor is above 1e-5.  That is the
  driven atmosphere after two steps: its horizontal momenta and horizontal B
  perturbations are second-order by-products of the vertical driver (1e-5 of
  the vertical momentum), shaped mostly by the hyperviscous cross terms, and
  the hyperviscosity coefficient -- a ratio of windowed maxima of third and
  first differences -- takes the FP32 rounding of the state into them: floor
  3.2e-5 on the horizontal momenta (3.3e-7 with hyperdiffusion off), 2.9e-5
  on the horizontal B.  Everywhere else the floor is ~1e-8 and the bar 1e-5;
* mixed under the dt rule: the same bar against the oracle run at the GPU's
  own dt sequence (the arithmetic at the same bar; a different dt alone moves
  the state by that relative amount times its change over the run), and
  every step's dt within 1e-2 of the oracle's.  The dt differs because the
  viscous limit divides by the largest hyperviscosity coefficient, formed
  from FP32 states; on smooth fields the third differences are small against
  q, so FP32 rounding of q moves the ratio.  Measured on a B200: the second
  step's dt 5.6e-3 off on the 256^2 vortex (its first step's coefficient
  comes from the smooth initial state) and 8.1e-4 from the third step on;
  5.1e-3 on the driven atmosphere's second step; 2e-5 on a 48^2 vortex.
"""
from __future__ import annotations

import numpy as np
import pytest

from smaug_b200 import PREC_FP64, PREC_MIXED, Batch, Engine, footprint, problems

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FP64_TOL, MIXED_TOL = 1e-6, 1e-5
NEAR_ZERO = 1e-9
FLOOR_FACTOR = 4.0


def field_errors(x, y, own: bool = False):
    """Per-field error of x against the reference y (inner cells, evolved
    fields), with the near-zero rule above; own=True gives every field's
    error against its own norm."""
    nw = 2 + 2 * (x.ndim - 1)
    sl = (slice(0, nw),) + tuple(slice(2, -2) for _ in range(x.ndim - 1))
    x, y = x[sl], y[sl]
    norms = np.array([np.linalg.norm(y[f]) for f in range(nw)])
    big = norms.max()
    out = []
    for f in range(nw):
        d = np.linalg.norm(x[f] - y[f])
        rel = norms[f] > (0.0 if own else NEAR_ZERO * big)
        out.append(d / norms[f] if rel else d / big)
    return np.array(out)


def _configs():
    return {
        "C1_ot256": (lambda: problems.orszag_tang(256), 10),
        "C2_blast128": (lambda: problems.blast_wave(128, seed=1234), 3),
        "C3_atmos256x128x128": (lambda: problems.atmosphere(256, 128, 128), 2),
    }


DT_RULE_TOL = 1e-2

_oracle_cache: dict = {}


def _oracle(name, make, steps, fixed: bool):
    """The oracle under the dt rule for `steps` RK4 steps -- (problem, state,
    per-step dts) -- or at a fixed dt of half the rule's last dt (one
    configuration cached at a time: the 3-D states are large)."""
    key = (name, fixed)
    if key not in _oracle_cache:
        rule = [v for k, v in _oracle_cache.items() if k == (name, False)]
        if fixed and not rule:
            _oracle(name, make, steps, False)
            rule = [_oracle_cache[(name, False)]]
        for k in [k for k in _oracle_cache if k[0] != name]:
            del _oracle_cache[k]
        prob = rule[0][0] if rule else make()
        dt0 = 0.5 * rule[0][2][-1] if fixed else 0.0
        o = Oracle(prob, dt_fixed=dt0)
        dts = []
        for _ in range(steps):
            o.step(1, rk4=True, dt_mode=0 if fixed else 1)
            dts.append(o.dt)
        _oracle_cache[key] = (prob, o.w.copy(), dts)
    return _oracle_cache[key]


def _oracle_at(prob, dts, fp32_state: bool = False):
    """The oracle stepped at a given per-step dt sequence; fp32_state rounds
    its evolved fields to FP32 after every step (the FP32 storage floor)."""
    o = Oracle(prob, dt_fixed=dts[0])
    nw = 2 + 2 * prob.ndim
    for dt in dts:
        o.s.dt = dt
        o.step(1, rk4=True, dt_mode=0)
        if fp32_state:
            o.w[:nw] = o.w[:nw].astype(np.float32).astype(np.float64)
    return o.w


@pytest.mark.parametrize("mode", ["fp64-dt_rule", "mixed-fixed_dt", "mixed-dt_rule"])
@pytest.mark.parametrize("name", list(_configs()))
def test_production_kernel_vs_oracle_at_config_size(need_gpu, name, mode):
    make, steps = _configs()[name]
    prec = PREC_FP64 if mode.startswith("fp64") else PREC_MIXED
    fixed = mode.endswith("fixed_dt")
    prob, w_ref, dts_ref = _oracle(name, make, steps, fixed)
    kw = {"dt_mode": 0, "dt0": dts_ref[0]} if fixed else {}
    e = Engine(prob, rk4=True, precision=prec, **kw)
    dts = []
    for _ in range(steps):
        e.step(1)
        dts.append(e.scalars()["dt"])
    e.sync()
    w = e.state()
    e.close()
    dt_tol = 1e-9 if prec == PREC_FP64 else DT_RULE_TOL
    dt_err = [abs(a - b) / b for a, b in zip(dts, dts_ref)]
    tol = np.full(2 + 2 * prob.ndim, FP64_TOL)
    floor = None
    if prec == PREC_MIXED:
        if not fixed:
            # the arithmetic at the GPU's own dt sequence
            w_ref = _oracle_at(prob, dts)
        floor = field_errors(_oracle_at(prob, dts, fp32_state=True), w_ref)
        tol = np.maximum(MIXED_TOL, FLOOR_FACTOR * floor)
    err = field_errors(w, w_ref)
    report = (name, mode, err, tol, floor, field_errors(w, w_ref, own=True), dt_err)
    assert np.all(err <= tol) and max(dt_err) <= dt_tol, report


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
    w = b.state(s_big)
    dt = b.scalars(s_big)["dt"]
    b.close()
    err = field_errors(w, o.w)
    tol = FP64_TOL if prec == PREC_FP64 else MIXED_TOL
    assert np.all(err <= tol), (err, field_errors(w, o.w, own=True))
    assert abs(dt - o.dt) <= 1e-9 * o.dt
