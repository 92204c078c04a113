"""The stratified atmosphere's background against the reference's own
helpers (CPU only).

The reference's spicule model builds its stratified background with two
helpers in models/initialisation_user.h.spicule1_mpi: temp() (345-360), the
tanh temperature profile, and inte() (326-343), the trapezoid rule of its
pressure integral.  oracle/ref_shim/build_ref.py cuts both out of the model
file and compiles them as they stand (oracle/_ref/libsmaug_ref_hydro.so).
problems.temperature_profile and problems.trapezoid_up restate them in the
same operation order, so they must give the same bits: the profile with the
model's own constants (T_ch = 15e3 K, T_co = 3e6 K, 2 Mm, 200 km), and the
running integral of 1 / lambda over the grid of the C3 atmosphere."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

from smaug_b200 import problems

LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libsmaug_ref_hydro.so"
pytestmark = pytest.mark.skipif(not LIB.exists(), reason="reference host build not present")

_PD = ctypes.POINTER(ctypes.c_double)


def _lib():
    L = ctypes.CDLL(str(LIB))
    L.ref_inte.argtypes = [_PD, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    L.ref_inte.restype = ctypes.c_double
    L.ref_temp.argtypes = [_PD, ctypes.c_int, _PD]
    return L


def _grid(nz=256, lz=6.0e6):
    dz = lz / nz
    n = nz + 4
    return -2 * dz + np.arange(n) * dz, dz


def test_temperature_profile_bits_equal_reference_temp():
    L = _lib()
    z, _ = _grid()
    T_ref = np.zeros_like(z)
    L.ref_temp(z.ctypes.data_as(_PD), len(z), T_ref.ctypes.data_as(_PD))
    T = problems.temperature_profile(z, t_ch=15.0e3, t_co=3.0e6, z_tr=2.0e6, w_tr=200.0e3)
    assert np.array_equal(T, T_ref)


def test_trapezoid_bits_equal_reference_inte():
    L = _lib()
    z, dz = _grid()
    T = problems.temperature_profile(z)
    inv = 1.0 / (-problems.R_GAS * T / problems.G_SUN)
    i0 = 2  # z = 0
    ours = problems.trapezoid_up(inv, i0, dz)
    col = np.ascontiguousarray(inv[i0:])
    for m in list(range(1, 12)) + [100, 150, len(col) - 1]:
        ref = L.ref_inte(col.ctypes.data_as(_PD), m + 1, 1, dz)
        assert ours[i0 + m] == ref, m


def test_atmosphere_background_is_hydrostatic():
    """rho_b of the C3 atmosphere: rho_b = rho0 at z = 0, and the pressure
    p_b = rho_b R T falls by exp(-int dz/lambda) between neighbouring points
    (the trapezoid rule of the reference's inte)."""
    prob = problems.atmosphere(64, 16)
    ids = problems.field_ids(2)
    rhob = prob.w[ids["rhob"], 0, :]
    z = prob.xmin[0] + np.arange(prob.n[0]) * prob.dx[0]
    T = problems.temperature_profile(z)
    assert rhob[2] == pytest.approx(2.7e-4, rel=1e-15)
    p = rhob * problems.R_GAS * T
    inv = 1.0 / (-problems.R_GAS * T / problems.G_SUN)
    ratio = p[3:] / p[2:-1]
    assert np.allclose(ratio, np.exp(-0.5 * (inv[2:-1] + inv[3:]) * prob.dx[0]), rtol=1e-13, atol=0)
