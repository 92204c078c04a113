"""CUDA path against the oracle and the golden fixtures (needs a GPU).

Bar: the FMA-free build (exact=True) must reproduce the oracle -- and so the
reference -- bit for bit; the production build (FMA contraction) must stay
within a relative L2 of 1e-6 per field after the stated number of steps.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

from smaug_b200 import Engine, problems

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"
sys.path.insert(0, str(GOLD))
from make_golden import CASES, make_problem, states_match  # noqa: E402

from oracle.oracle import Oracle  # noqa: E402

pytestmark = pytest.mark.gpu

# FMA contraction changes last bits; the reference's viscous-dt rule takes a
# running maximum of a hyperviscosity that is driven by rounding noise in flat
# regions, so dt (and then the state) moves by ~1e-8 relative within a few
# steps.  The CPU oracle built with FMA contraction shows the same spread
# against the FMA-free oracle.  Bar: 1e-6 (the method target is 1e-5).
FAST_RTOL = 1e-6


def rel_l2(a, b):
    """Per-field relative L2 over inner cells (absolute where the field is 0)."""
    out = []
    sl = (slice(None),) + tuple(slice(2, -2) for _ in range(a.ndim - 1))
    a, b = a[sl], b[sl]
    for f in range(a.shape[0]):
        nb = np.linalg.norm(b[f])
        out.append(np.linalg.norm(a[f] - b[f]) / (nb if nb > 0 else 1.0))
    return np.array(out)


@pytest.mark.parametrize("name", sorted(CASES))
def test_exact_build_reproduces_golden(need_gpu, name):
    meta = json.loads((GOLD / f"{name}.json").read_text())
    spec = meta["spec"]
    gold = np.load(GOLD / f"{name}.npz")
    prob = make_problem(spec)
    eng = Engine(prob, rk4=spec["rk4"], exact=True)
    dts = []
    for _ in range(spec["steps"]):
        eng.step(1)
        dts.append(eng.scalars()["dt"])
    eng.sync()
    w = eng.state()
    assert np.array_equal(np.array(dts), gold["dts"]), (dts, gold["dts"])
    assert states_match(w, gold["w_final"], spec, meta["source"]), rel_l2(w, gold["w_final"])


@pytest.mark.parametrize("kind,n,btype,rk4,steps", [
    ("ot", 48, None, True, 12),
    ("ot", 40, (4, 0), True, 8),
    ("ot", 36, (0, 4), False, 10),
    ("blast", 16, None, True, 5),
    ("blast", 14, (0, 0, 4), True, 4),
])
def test_exact_build_bit_exact_vs_oracle(need_gpu, kind, n, btype, rk4, steps):
    prob = problems.orszag_tang(n) if kind == "ot" else problems.blast_wave(n, seed=11)
    if btype:
        prob.btype = btype
    o = Oracle(prob)
    eng = Engine(prob, rk4=rk4, exact=True)
    for s in range(steps):
        o.step(1, rk4=rk4)
        eng.step(1)
        sc = eng.scalars()
        assert sc["dt"] == o.dt, (s, sc["dt"], o.dt)
    w = eng.state()
    assert np.array_equal(w, o.w), rel_l2(w, o.w)
    assert eng.scalars()["maxviscoef"] == o.s.maxviscoef


@pytest.mark.parametrize("kind,n,steps", [("ot", 64, 40), ("blast", 20, 10)])
def test_fast_build_within_tolerance(need_gpu, kind, n, steps):
    prob = problems.orszag_tang(n) if kind == "ot" else problems.blast_wave(n)
    o = Oracle(prob)
    o.step(steps, rk4=True)
    eng = Engine(prob, rk4=True, exact=False)
    eng.step(steps)
    eng.sync()
    err = rel_l2(eng.state(), o.w)
    assert np.all(err < FAST_RTOL), err


@pytest.mark.parametrize("rk4", [False, True])
def test_exact_build_atmosphere_with_timed_driver(need_gpu, rk4):
    """Stratified atmosphere (gravity, contcd4, backgrounds) with the default
    sinusoidal driver: the FMA-free build against the oracle.  The driver's
    sin() comes from CUDA on the device and from libm in the oracle, so the
    bar here is a relative L2 of 1e-13 rather than bit equality (the same
    case with a constant driver is bit-exact: atmos40x20_drv_rk4)."""
    prob = problems.atmosphere(40, 20, noise=1e-3, seed=5)
    prob.driver["amp"] = 2.0e3
    prob.driver["period"] = 2.0  # several periods within the run
    o = Oracle(prob)
    eng = Engine(prob, rk4=rk4, exact=True)
    for _ in range(6):
        o.step(1, rk4=rk4)
        eng.step(1)
    err = rel_l2(eng.state(), o.w)
    assert np.all(err < 1e-13), err
    assert abs(eng.scalars()["dt"] - o.dt) <= 1e-13 * o.dt


@pytest.mark.parametrize("precision,tol", [(0, FAST_RTOL), (1, 1e-5)])
def test_fast_build_atmosphere_with_driver(need_gpu, precision, tol):
    prob = problems.atmosphere(48, 24, noise=1e-3, seed=6)
    prob.driver["amp"] = 2.0e3
    prob.driver["period"] = 3.0
    o = Oracle(prob)
    o.step(8, rk4=True)
    eng = Engine(prob, rk4=True, precision=precision)
    eng.step(8)
    err = rel_l2(eng.state(), o.w)
    assert np.all(err < tol), err


def test_device_pointer_state_roundtrip(need_gpu):
    import torch
    prob = problems.orszag_tang(32)
    eng = Engine(prob, rk4=True)
    w = torch.from_numpy(np.ascontiguousarray(prob.w)).cuda()
    eng.set_state_device(w.data_ptr(), w.numel())
    eng.step(2)
    out = torch.empty_like(w)
    eng.get_state_device(out.data_ptr(), out.numel())
    eng.sync()
    ref = Engine(prob, rk4=True)
    ref.step(2)
    assert np.array_equal(out.cpu().numpy(), ref.state())


def test_bad_sizes_are_rejected(need_gpu):
    from smaug_b200 import SmaugError
    prob = problems.orszag_tang(16)
    eng = Engine(prob)
    with pytest.raises(SmaugError):
        eng.set_state(prob.w[:5])
