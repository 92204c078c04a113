"""The reference's single-step host loop (host/ref_loop.c: the call sequence
of iosmaug.cpp:783-1166 with rkon = 0 and moddton = 1) driven through the
reference-compatible per-operator entry points (libsmaug_cu2d.so,
libsmaug_cu3d.so), against the CPU oracle's single step on the same state
(needs a GPU).  The entry points are built without FMA contraction and
restate the reference's arithmetic per operator, so the loop must give the
oracle's bits -- and so the reference's."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from smaug_b200 import problems, vacio
from smaug_b200.build import ref_loop_exe

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _run_loop(tmp_path, prob, steps, *opts):
    cfg = tmp_path / "in.ini"
    vacio.write_ascii(cfg, vacio.header_for(prob), vacio.positions(prob), prob.w)
    out = tmp_path / "out.out"
    r = subprocess.run([str(ref_loop_exe(prob.ndim)), str(cfg), str(steps), str(out), *opts], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    _, _, w = vacio.read_binary(out)
    dt = float(r.stdout.split()[1])
    return w, dt


@pytest.mark.parametrize("case", ["ot", "ot_cd4x", "ot_divb", "blast", "blast_cd4z", "ot_nohyper"])
def test_reference_loop_through_shims_bits_equal_oracle(need_gpu, tmp_path, case):
    opts = []
    if case.startswith("ot"):
        prob = problems.orszag_tang(32, rho_noise=0.01, seed=2)
    else:
        prob = problems.blast_wave(12, seed=7)
    if case == "ot_cd4x":
        prob.btype = (4, 0)
        opts = ["--btype", "4,0"]
    if case == "blast_cd4z":
        prob.btype = (0, 0, 4)
        opts = ["--btype", "0,0,4"]
    if case == "ot_divb":
        prob.divb = 1
        opts = ["--divb"]
    if case == "ot_nohyper":
        prob.hyperdif = 0
        opts = ["--no-hyperdif"]
    steps = 5
    w, dt = _run_loop(tmp_path, prob, steps, *opts)
    o = Oracle(prob)
    o.step(steps, rk4=False)
    assert dt == o.dt
    assert np.array_equal(w, o.w), np.abs(w - o.w).max()
