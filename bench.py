#!/usr/bin/env python3
"""Benchmark: ideal-MHD cell-updates/s on B200 (SAC/SMAUG method).

Workload (one step = one full RK4 step of the whole grid): the 3-D blast wave,
128^3 interior cells (+2 ghost layers), periodic, hyperdiffusion on, Courant
0.3 with the reference's dt rule; seeded synthetic initial state.  The
headline line runs the mixed-precision path (FP32 stage states and stencils,
FP64 backgrounds, pressure / internal-energy recovery, RK base and sum, dt);
the plain FP64 path is measured beside it on the same workload ("companion")
and the two final states are compared ("accuracy").
With --gpus N (torchrun) every rank advances its own replica (no data-path
collective: independent instances), so scaling is weak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision mixed|fp64]

--impl reference times the reference's own CPU implementation (the SMAUG
sources built for the host, oracle/_ref) on a bounded sample of the same
workload using every host core (one reference process per core).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "smaug-all_b200" / "python"))

METRIC = "cell-updates/s (3-D blast wave 128^3, RK4; mixed FP32/FP64 vs plain FP64)"
UNIT = "cell-updates/s"
# algorithmic HBM bytes per cell-update (one cell, one full RK4 step), 3-D:
# FP64: 14 evolved-field passes x 8 fields x 8 B + 4 background passes x 5 x 8 B
BYTES_PER_CELL_UPDATE_FP64_3D = (14 * 8 + 4 * 5) * 8  # 1056 B
# mixed: 19 FP32 evolved-field passes x 8 fields x 4 B + 4 FP64 background passes
BYTES_PER_CELL_UPDATE_MIXED_3D = 19 * 8 * 4 + 4 * 5 * 8  # 768 B
SAMPLE_N = 24          # CPU sample: 24^3 interior cells per process
SAMPLE_SUBSTEPS = 4    # reference single steps per RK4-equivalent step


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per stage launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "stage_kernel_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return None
    return None


# ----------------------------------------------------------------- CPU side

def _cpu_worker(args):
    n, substeps, nsteps, warmup, use_ref = args
    # the reference's host code prints progress on stdout; keep the bench's
    # stdout to its one JSON line
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    import numpy as np  # noqa: F401
    from smaug_b200 import problems
    prob = problems.blast_wave(n)
    if use_ref:
        from oracle.oracle import Reference
        sim = Reference(prob)
        sim.step(warmup * substeps)
        t = time.perf_counter()
        for _ in range(nsteps):
            sim.step(substeps)
    else:
        from oracle.oracle import Oracle
        sim = Oracle(prob)
        sim.step(warmup, rk4=True)
        t = time.perf_counter()
        sim.step(nsteps, rk4=True)
    return time.perf_counter() - t


def cpu_throughput(nsteps: int, warmup: int = 1, procs: int | None = None):
    """Cell-updates/s of the reference's CPU code on the host cores."""
    import multiprocessing as mp
    use_ref = (ROOT / "oracle" / "_ref" / "libsmaug_ref3d.so").exists()
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    substeps = SAMPLE_SUBSTEPS if use_ref else 1
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        times = pool.map(_cpu_worker, [(SAMPLE_N, substeps, nsteps, warmup, use_ref)] * procs)
    wall = time.perf_counter() - t0
    elapsed = max(times)
    cells = SAMPLE_N ** 3
    value = procs * cells * nsteps / elapsed
    kind = "reference" if use_ref else "port"
    sample = (f"{procs} processes x blast wave {SAMPLE_N}^3 x {nsteps} RK4-equivalent steps "
              + (f"({substeps} reference single steps each; reference rkon=1 path is not usable)" if use_ref
                 else "(oracle port, RK4)"))
    return {"value": value, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample,
            "elapsed_s": elapsed, "wall_s": wall}


def run_reference(a):
    """The reference arm: the reference's CPU code on every host core."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cpu = cpu_throughput(nsteps=max(1, a.steps), warmup=max(1, a.warmup))
    line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": cpu["elapsed_s"] * 1e3 / max(1, a.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": dict(workload_config(a.n, a.gpus), precision="fp64 (the reference computes in FP64 only)"),
            "impl": "reference",
            "cpu_baseline": {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": cpu["kind"],
                             "sample": cpu["sample"]},
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def workload_config(n: int, world: int, ncells: int | None = None):
    ncells = ncells or (n + 4) ** 3
    return {"workload": f"blast wave 3-D {n}^3 interior, periodic, RK4, hyperdiffusion on",
            "ndim": 3, "interior": [n] * 3, "cells_with_ghosts": ncells,
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2: state 4 x 8 fields x {ncells} x 8 B = "
                  f"{4 * 8 * ncells * 8 / 1e6:.0f} MB > 126 MB"}


# ----------------------------------------------------------------- GPU side

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = ROOT / "gpurun_out" / f"clocks_rank{device}.csv"

    def start(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        sm = sorted(r[0] for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": rows[0][1], "reasons": reasons, "samples": len(rows)}


def measure(eng, n_int, steps, warmup, stream, barrier, dist, world, local, sample_clocks):
    """Device-timed throughput of `steps` full steps of one engine, plus the
    average duration of its stage-kernel launches."""
    import torch
    eng.step(max(3, warmup))
    eng.sync()
    sampler = ClockSampler(local) if sample_clocks else None
    if sampler:
        sampler.start()
    barrier()
    torch.cuda.synchronize()
    l0 = eng.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.step(steps)
    ev1.record(stream)
    eng.sync()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if sampler else None
    ms = ev0.elapsed_time(ev1)
    launches = eng.launches - l0
    t = torch.tensor([ms], device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    # per-launch duration of the stage kernel (the dominant kernel)
    eng.profile_stages(True)
    eng.step(max(2, min(steps, 8)))
    st_ms, st_n = eng.stage_times()
    eng.profile_stages(False)
    return {"value": world * n_int * steps / (ms_max / 1e3), "ms_per_step": ms_max / steps,
            "launches": launches, "clocks": clocks, "avg_stage_ms": st_ms / max(st_n, 1)}


def accuracy_study(prob, steps: int, device: int):
    """Per-field relative L2 (inner cells) of the mixed and the FP64-FMA
    states against the FMA-free FP64 build after `steps` RK4 steps, under the
    reference's dt rule and at a fixed dt."""
    import numpy as np

    from smaug_b200 import PREC_MIXED, Engine

    def rel(w, ref, nw):
        sl = (slice(0, nw),) + (slice(2, -2),) * (w.ndim - 1)
        x, y = w[sl], ref[sl]
        norms = np.array([np.linalg.norm(y[f]) for f in range(nw)])
        return [float(np.linalg.norm(x[f] - y[f]) / (norms[f] if norms[f] > 0 else norms.max())) for f in range(nw)]

    nw = 2 + 2 * prob.ndim
    out = {"steps": steps, "reference": "FP64 FMA-free build (bit-identical to the oracle)"}
    dt_fixed = None
    for mode in ("dt_rule", "fixed_dt"):
        kw = {"dt_mode": 1} if mode == "dt_rule" else {"dt_mode": 0, "dt0": dt_fixed}
        ex = Engine(prob, rk4=True, exact=True, device=device, **kw)
        fa = Engine(prob, rk4=True, device=device, **kw)
        mi = Engine(prob, rk4=True, device=device, precision=PREC_MIXED, **kw)
        for e in (ex, fa, mi):
            e.step(steps)
        we = ex.state()
        rm, rf = rel(mi.state(), we, nw), rel(fa.state(), we, nw)
        out[mode] = {"mixed_max_rel_l2": max(rm), "mixed_rel_l2_per_field": rm, "fp64_fma_max_rel_l2": max(rf)}
        if mode == "dt_rule":
            dt_fixed = 0.5 * ex.scalars()["dt"]
        else:
            out[mode]["dt"] = dt_fixed
        for e in (ex, fa, mi):
            e.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128, help="interior cells per dim")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="arithmetic of the headline line (the other one is measured beside it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-companion", action="store_true", help="skip the other precision's measurement")
    ap.add_argument("--accuracy-steps", type=int, default=50,
                    help="steps of the accuracy study against the FP64 oracle (0: skip)")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference(a)

    import ctypes

    import numpy as np
    import torch

    from smaug_b200 import PREC_FP64, PREC_MIXED, Engine, problems

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    prob = problems.blast_wave(a.n, seed=1234 + rank)
    n_int = prob.interior
    mixed = a.precision == "mixed"
    prec = PREC_MIXED if mixed else PREC_FP64
    eng = Engine(prob, rk4=True, exact=False, device=local, precision=prec)
    stream = torch.cuda.ExternalStream(eng.stream)

    # ---- headline: K steps, device time on the engine's stream
    m = measure(eng, n_int, a.steps, a.warmup, stream, barrier, dist, world, local, sample_clocks=True)
    alg_bytes_per_launch = (BYTES_PER_CELL_UPDATE_MIXED_3D if mixed else BYTES_PER_CELL_UPDATE_FP64_3D) / 4 * n_int
    achieved = alg_bytes_per_launch / (m["avg_stage_ms"] / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    tr = load_traffic()
    traffic = None
    kernel = f"tile_stage_kernel<3,{'float' if mixed else 'double'}>"
    if tr and tr.get(kernel, {}).get("n") == a.n:
        traffic = tr[kernel].get("dram_bytes_per_launch")

    # ---- the other precision on the same workload
    companion = None
    if not a.no_companion:
        eng2 = Engine(prob, rk4=True, exact=False, device=local, precision=PREC_FP64 if mixed else PREC_MIXED)
        s2 = torch.cuda.ExternalStream(eng2.stream)
        m2 = measure(eng2, n_int, a.steps, a.warmup, s2, barrier, dist, world, local, sample_clocks=False)
        companion = {"precision": "fp64" if mixed else "mixed", "value": m2["value"],
                     "ms_per_step": m2["ms_per_step"], "avg_stage_ms": m2["avg_stage_ms"]}
        eng2.close()

    # ---- accuracy against the FP64 oracle (the FMA-free FP64 build, which
    # reproduces it bit for bit), beside the drift of the FP64 FMA build
    accuracy = None
    if a.accuracy_steps > 0 and rank == 0:
        accuracy = accuracy_study(prob, a.accuracy_steps, local)

    # ---- end to end through the public C ABI with host buffers: every step
    # uploads its input state from pinned host memory (smaug_set_state),
    # advances one step (smaug_step) and reads the new state and the step's
    # scalars back (smaug_get_state, smaug_get_scalars)
    dptr = ctypes.POINTER(ctypes.c_double)
    host = torch.from_numpy(np.ascontiguousarray(prob.w)).pin_memory()
    host_p = host.numpy().ctypes.data_as(dptr)
    scal = (ctypes.c_double * 8)()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(a.steps):
        eng.lib.smaug_set_state(eng.h, host_p, host.numel())
        eng.lib.smaug_step(eng.h, 1)
        eng.lib.smaug_get_state(eng.h, host_p, host.numel())
        eng.lib.smaug_get_scalars(eng.h, scal)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    te = torch.tensor([e2e_ms], device="cuda")
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * n_int * a.steps / (float(te.item()) / 1e3)
    state_bytes = host.numel() * 8

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            cpu = cpu_throughput(nsteps=2, warmup=1)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # the GPU number stands on its own
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        cfg = workload_config(a.n, world, prob.ncells)
        cfg["precision"] = "mixed: FP32 states/stencils, FP64 p_T, e_int, base, RK sum, dt" if mixed else "fp64"
        line = {
            "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": max(3, a.warmup), "ms_per_step": m["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": kernel, "avg_launch_ms": m["avg_stage_ms"],
                         "alg_bytes_per_launch": alg_bytes_per_launch},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes + 8 * 8},
            "gpu_launches": m["launches"],
            "clocks": m["clocks"],
        }
        if companion:
            line["companion"] = companion
            line["mixed_vs_fp64"] = (m["value"] / companion["value"]) if mixed else (companion["value"] / m["value"])
        if accuracy:
            line["accuracy"] = accuracy
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
