"""The C host driver (host/smaug_run.c, built by build() beside the
library): a C program that reads a VAC configuration file, derives the metric
with smaug_initgrid, runs the step loop through the C ABI stage by stage on
its own CUDA stream and writes VAC snapshots -- the shape of the reference's
host loop (iosmaug.cpp:802-1166) -- compared with the oracle on the same
state (needs a GPU).  The FMA-free build must give the oracle's bits."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from smaug_b200 import problems, vacio
from smaug_b200.build import HOST_EXE

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _run(tmp_path, prob, steps, *opts):
    cfg = tmp_path / "in.ini"
    vacio.write_ascii(cfg, vacio.header_for(prob), vacio.positions(prob), prob.w)
    out = tmp_path / "snap"
    r = subprocess.run([str(HOST_EXE), str(cfg), str(steps), str(out), *opts], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return out, r.stdout


@pytest.mark.parametrize("rk4", [True, False])
def test_host_driver_exact_build_bits_equal_oracle(need_gpu, tmp_path, rk4):
    prob = problems.orszag_tang(48, rho_noise=0.01, seed=9)
    steps = 6
    out, _ = _run(tmp_path, prob, steps, "--exact", *([] if rk4 else ["--single"]))
    h, pos, w = vacio.read_binary(f"{out}_{steps}.out")
    o = Oracle(prob)
    t = 0.0
    for _ in range(steps):
        o.step(1, rk4=rk4)
        t += o.dt
    assert h["it"] == steps and h["t"] == pytest.approx(t, rel=1e-14)
    assert np.array_equal(pos, vacio.positions(prob))
    assert np.array_equal(w, o.w)


def test_host_driver_production_and_snapshots(need_gpu, tmp_path):
    prob = problems.orszag_tang(64, rho_noise=0.01, seed=10)
    out, stdout = _run(tmp_path, prob, 5, "--save-every", "2")
    assert "5 steps" in stdout
    # snapshots of the state before steps 1, 3, 5 and the final one
    for it in (0, 2, 4, 5):
        assert (tmp_path / f"snap_{it}.out").exists(), it
    _, _, w0 = vacio.read_binary(f"{out}_0.out")
    o = Oracle(prob)
    assert np.array_equal(w0, o.w)  # the loaded state with its ghosts filled
    o.step(5, rk4=True)
    _, _, w = vacio.read_binary(f"{out}_5.out")
    sl = (slice(0, 6), slice(2, -2), slice(2, -2))
    err = max(np.linalg.norm(w[sl][f] - o.w[sl][f]) / np.linalg.norm(o.w[sl][f]) for f in range(6))
    assert err <= 1e-6, err
