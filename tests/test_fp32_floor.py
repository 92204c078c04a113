"""The FP32 storage floor of the driven atmosphere (CPU, oracle only).

The mixed path stores its stage states in FP32.  What that alone costs is
measured by the FP64 oracle whose evolved state is rounded to FP32 after every
step: the floor that the config-size parity bar of the mixed path is scaled
from.  On the driven atmosphere after two steps the floor of the horizontal
momentum -- a second-order by-product of the vertical driver -- is far above
FP32 rounding, and it comes from the hyperviscosity: the coefficient is a
ratio of windowed maxima of third and first differences, which carries the
state's rounding into the by-product fields.  With hyperdiffusion off the
same rounding leaves them near FP32 resolution.  The dense fields (rho, the
vertical momentum, e) stay at FP32 resolution either way.
"""
from __future__ import annotations

import numpy as np

from smaug_b200 import problems

from oracle.oracle import Oracle


def _floor(hyperdif: int):
    prob = problems.atmosphere(256, 128)
    prob.hyperdif = hyperdif
    probe = Oracle(prob)
    probe.step(1, rk4=True)
    dt = 0.5 * probe.dt
    ref, fl = Oracle(prob, dt_fixed=dt), Oracle(prob, dt_fixed=dt)
    for _ in range(2):
        ref.step(1, rk4=True, dt_mode=0)
        fl.step(1, rk4=True, dt_mode=0)
        fl.w[:6] = fl.w[:6].astype(np.float32).astype(np.float64)
    sl = (slice(0, 6), slice(2, -2), slice(2, -2))
    x, y = fl.w[sl], ref.w[sl]
    return np.array([np.linalg.norm(x[f] - y[f]) / np.linalg.norm(y[f]) for f in range(6)])


def test_fp32_storage_floor_comes_from_the_hyperviscosity():
    on, off = _floor(1), _floor(0)
    # fields: rho, m_z (driven), m_x (by-product), e, B_z, B_x
    for f in (0, 1, 3):
        assert on[f] < 1e-7 and off[f] < 1e-7, (f, on, off)
    assert on[2] > 1e-5, on  # 2.3e-5 measured
    assert off[2] < 1e-6, off  # 3.0e-7 measured
    assert on[2] > 30 * off[2], (on, off)
