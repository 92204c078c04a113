"""Mixed-precision path (FP32 stage states and stencils, FP64 where accuracy
needs it) against the FP64 oracle and the FP64 CUDA path (needs a GPU).

Error measure: per field, the relative L2 norm over inner cells,
||x - x_ref||_2 / ||x_ref||_2; a field whose reference norm is 0 is measured
absolutely and normalised by the largest norm of the other fields.  Bar: 1e-5
per field, the stated tolerance for FP32-bulk / FP64-critical runs.

The method amplifies rounding differences: the hyperviscosity coefficient is a
ratio of windowed maxima of third and first differences, and the viscous dt
takes the running maximum of that coefficient.  Two FP64 builds that differ
only in FMA contraction drift apart to ~1e-2 relative L2 within 1000 steps of
an Orszag-Tang vortex (and within 500 steps of the blast wave under the dt
rule).  So the 1e-5 bar applies where the run does not amplify (fixed dt
without the chaotic switch regime, hyperdiffusion off, or short horizons), and
over long amplifying runs the mixed path is held to the FP64-FMA drift.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import Oracle
from smaug_b200 import PREC_MIXED, Engine, SmaugError, problems

pytestmark = pytest.mark.gpu

MIXED_RTOL = 1e-5
# long amplifying runs: mixed drift at most this multiple of the drift of the
# FP64 FMA build (both measured against the FMA-free FP64 build); measured
# 3.7x on the 96^2 Orszag-Tang vortex after 1000 steps (2.1e-2 against 5.7e-3)
DRIFT_FACTOR = 5.0


def field_errors(w, ref, nw):
    sl = (slice(None),) + tuple(slice(2, -2) for _ in range(w.ndim - 1))
    a, b = w[sl][:nw], ref[sl][:nw]
    norms = np.array([np.linalg.norm(b[f]) for f in range(nw)])
    scale = norms.max()
    return np.array([np.linalg.norm(a[f] - b[f]) / (norms[f] if norms[f] > 0 else scale) for f in range(nw)])


def nw_of(prob):
    return 2 + 2 * prob.ndim


@pytest.mark.parametrize("kind,n,steps,dt_mode,dt0", [
    ("ot", 48, 5, 1, 0.0),       # short horizon under the reference's dt rule
    ("ot", 48, 80, 1, 0.0),      # hyperdiffusion off below
    ("blast", 16, 40, 0, 2e-4),  # fixed dt
])
def test_mixed_vs_oracle(need_gpu, kind, n, steps, dt_mode, dt0):
    prob = problems.orszag_tang(n) if kind == "ot" else problems.blast_wave(n, seed=5)
    if kind == "ot" and steps > 5:
        prob.hyperdif = 0
    o = Oracle(prob, dt_fixed=dt0)
    o.step(steps, rk4=True, dt_mode=dt_mode)
    eng = Engine(prob, rk4=True, precision=PREC_MIXED, dt_mode=dt_mode, dt0=dt0)
    eng.step(steps)
    eng.sync()
    err = field_errors(eng.state(), o.w, nw_of(prob))
    assert err.max() <= MIXED_RTOL, err
    # the FP32 path really is a different computation, not the FP64 one
    assert err.max() > 0.0
    # Under the dt rule with hyperdiffusion on, dt is the viscous limit. It is
    # inversely proportional to the largest hyperviscosity coefficient, i.e. to
    # max|d3 q| / max|d1 q| with q in FP32. Rounding q (6e-8 relative) puts up
    # to 8 x 6e-8 |q| into a third difference of size (k dx)^3 |q| ~ 3e-3 |q|
    # on a 48^2 Orszag-Tang grid: 1.6e-4 relative. The Courant limit carries
    # only the wave speeds' FP32 rounding.
    viscous = dt_mode == 1 and prob.hyperdif and o.s.dtdiffvisc == o.dt
    dt_rtol = 2e-4 if viscous else 1e-5
    assert abs(eng.scalars()["dt"] - o.dt) <= dt_rtol * o.dt


def test_mixed_blast_500_steps_fixed_dt(need_gpu):
    """Blast wave, 500 RK4 steps at fixed dt, hyperdiffusion on: mixed against
    the FP64 path's FMA-free build (bit-identical to the oracle)."""
    prob = problems.blast_wave(32, seed=5)
    ref = Engine(prob, rk4=True, exact=True, dt_mode=0, dt0=2e-4)
    mix = Engine(prob, rk4=True, precision=PREC_MIXED, dt_mode=0, dt0=2e-4)
    ref.step(500)
    mix.step(500)
    err = field_errors(mix.state(), ref.state(), nw_of(prob))
    assert err.max() <= MIXED_RTOL, err


def test_mixed_long_run_drift_within_fp64_rounding_drift(need_gpu):
    """1000 RK4 steps of a 2-D Orszag-Tang vortex under the reference's dt
    rule: the mixed path's drift from the FMA-free FP64 build stays within
    DRIFT_FACTOR times the drift of the FP64 FMA build."""
    prob = problems.orszag_tang(96)
    ref = Engine(prob, rk4=True, exact=True)
    fma = Engine(prob, rk4=True)
    mix = Engine(prob, rk4=True, precision=PREC_MIXED)
    for e in (ref, fma, mix):
        e.step(1000)
    wr = ref.state()
    e_fma = field_errors(fma.state(), wr, nw_of(prob)).max()
    e_mix = field_errors(mix.state(), wr, nw_of(prob)).max()
    assert np.isfinite(e_mix) and e_mix <= DRIFT_FACTOR * e_fma, (e_mix, e_fma)


def test_mixed_state_roundtrip_is_lossless(need_gpu):
    """Loading a state splits it into FP32 value + compensation; reading it
    back before any step returns the FP64 input to the last bit or two."""
    prob = problems.blast_wave(12, seed=3)
    eng = Engine(prob, rk4=True, precision=PREC_MIXED)
    w = eng.state()
    ref = Engine(prob, rk4=True).state()  # ghost-filled FP64 input
    rel = np.abs(w - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() <= 2.0 ** -46, rel.max()


def test_mixed_rejects_single_step_and_exact(need_gpu):
    prob = problems.orszag_tang(24)
    with pytest.raises(SmaugError):
        Engine(prob, rk4=False, precision=PREC_MIXED)
    with pytest.raises(SmaugError):
        Engine(prob, rk4=True, exact=True, precision=PREC_MIXED)
