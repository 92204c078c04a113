#!/usr/bin/env python3
"""Regenerate the golden fixtures in tests/golden/ (run in the build container,
where the reference sources exist and oracle/ref_shim/build_ref.py can build
the host version of the reference).

Single-step fixtures come from the reference itself (oracle/_ref): the
reference's own cu* sequence of dev/smaug/src/iosmaug.cpp:802-1166, moddton=1.
RK4 fixtures come from the oracle (the reference has no working RK4 path;
the oracle's single step equals the reference's bit for bit).

Each case runs in its own process because the reference library keeps one
global simulation.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "smaug-all_b200" / "python"))

CASES = {
    "ot24_euler": dict(kind="ot", n=24, btype=None, steps=6, rk4=False),
    "ot24_cd4x_euler": dict(kind="ot", n=24, btype=[4, 0], steps=6, rk4=False),
    "ot20_cd4y_euler": dict(kind="ot", n=20, btype=[0, 4], steps=5, rk4=False),
    "blast10_euler": dict(kind="blast", n=10, btype=None, steps=4, rk4=False),
    "blast10_cd4x_euler": dict(kind="blast", n=10, btype=[4, 0, 0], steps=3, rk4=False),
    "ot24_rk4": dict(kind="ot", n=24, btype=None, steps=4, rk4=True),
    "blast10_rk4": dict(kind="blast", n=10, btype=None, steps=3, rk4=True),
}


def make_problem(spec):
    from smaug_b200 import problems
    if spec["kind"] == "ot":
        prob = problems.orszag_tang(spec["n"])
    else:
        prob = problems.blast_wave(spec["n"])
    if spec.get("btype"):
        prob.btype = tuple(spec["btype"])
    return prob


def run_case(name: str) -> None:
    from oracle.oracle import Oracle, Reference
    spec = CASES[name]
    prob = make_problem(spec)
    dts, states = [], []
    if spec["rk4"]:
        o = Oracle(prob)
        for _ in range(spec["steps"]):
            o.step(1, rk4=True)
            dts.append(o.dt)
        states.append(o.w.copy())
        source = "oracle"
    else:
        r = Reference(prob)
        for _ in range(spec["steps"]):
            w = r.step(1)
            dts.append(r.dt)
        states.append(w.copy())
        source = "reference"
    np.savez_compressed(HERE / f"{name}.npz", w_final=states[-1], dts=np.array(dts))
    (HERE / f"{name}.json").write_text(json.dumps({"spec": spec, "source": source}, indent=1) + "\n")
    print(name, source, dts[-1])


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run_case(sys.argv[1])
    else:
        for n in CASES:
            subprocess.run([sys.executable, __file__, n], check=True, stdout=subprocess.PIPE)
            print("wrote", n)
