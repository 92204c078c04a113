#!/usr/bin/env python3
"""Benchmark: ideal-MHD cell-updates/s on B200 (SAC/SMAUG method).

Workload (one step = one full RK4 step of the whole grid): the 3-D blast wave,
128^3 interior cells (+2 ghost layers), periodic, FP64, hyperdiffusion on,
Courant 0.3 with the reference's dt rule; seeded synthetic initial state.
With --gpus N (torchrun) every rank advances its own replica (no data-path
collective: independent instances), so scaling is weak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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

METRIC = "cell-updates/s (3-D blast wave 128^3, RK4, FP64)"
UNIT = "cell-updates/s"
BYTES_PER_CELL_UPDATE_FP64_3D = (14 * 8 + 4 * 5) * 8  # 1056 B: RK4 minimum traffic
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
    n, substeps, nsteps, use_ref = args
    import numpy as np  # noqa: F401
    from smaug_b200 import problems
    prob = problems.blast_wave(n)
    if use_ref:
        from oracle.oracle import Reference
        sim = Reference(prob)
        sim.step(1)
        t = time.perf_counter()
        for _ in range(nsteps):
            sim.step(substeps)
    else:
        from oracle.oracle import Oracle
        sim = Oracle(prob)
        sim.step(1, rk4=True)
        t = time.perf_counter()
        sim.step(nsteps, rk4=True)
    return time.perf_counter() - t


def cpu_throughput(nsteps: int, procs: int | None = None):
    """Cell-updates/s of the reference's CPU code on the host cores."""
    import multiprocessing as mp
    use_ref = (ROOT / "oracle" / "_ref" / "libsmaug_ref3d.so").exists()
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    substeps = SAMPLE_SUBSTEPS if use_ref else 1
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        times = pool.map(_cpu_worker, [(SAMPLE_N, substeps, nsteps, use_ref)] * procs)
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
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    res = cpu_throughput(nsteps=a.warmup + a.steps) if False else None
    # warm-up and timed steps, each a bounded sample
    import multiprocessing as mp  # noqa: F401
    cpu = cpu_throughput(nsteps=max(1, a.steps))
    line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"blast wave 3-D, sample {SAMPLE_N}^3 per core", "ndim": 3,
                       "interior": [SAMPLE_N] * 3, "method": "SMAUG single step x4 per RK4-equivalent step"},
            "impl": "reference",
            "cpu_baseline": {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": cpu["kind"],
                             "sample": cpu["sample"]},
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    del res
    print(json.dumps(line))
    return 0


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128, help="interior cells per dim")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference(a)

    import numpy as np
    import torch

    from smaug_b200 import Engine, problems

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
    eng = Engine(prob, rk4=True, exact=False, device=local)
    n_int = prob.interior
    stream = torch.cuda.ExternalStream(eng.stream)

    eng.step(max(3, a.warmup))
    eng.sync()

    # ---- timed region: K steps, device time on the engine's stream
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    l0 = eng.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.step(a.steps)
    ev1.record(stream)
    eng.sync()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    launches = eng.launches - l0
    t = torch.tensor([ms], device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * n_int * a.steps / (ms_max / 1e3)

    # ---- per-launch duration of the stage kernel (dominant kernel)
    eng.profile_stages(True)
    eng.step(max(2, min(a.steps, 8)))
    st_ms, st_n = eng.stage_times()
    eng.profile_stages(False)
    avg_stage_ms = st_ms / max(st_n, 1)
    alg_bytes_per_launch = BYTES_PER_CELL_UPDATE_FP64_3D / 4 * n_int
    achieved = alg_bytes_per_launch / (avg_stage_ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    tr = load_traffic()
    traffic = None
    if tr and tr.get("n") == a.n:
        traffic = tr.get("dram_bytes_per_launch")

    # ---- end to end through the public API with host buffers
    host = torch.from_numpy(np.ascontiguousarray(prob.w)).pin_memory()
    host_out = torch.empty_like(host).pin_memory()
    scal = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    eng.lib.smaug_set_state(eng.h, host.numpy().ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)), host.numel())
    for _ in range(a.steps):
        eng.step(1)
        scal.append(eng.scalars()["dt"])
    eng.lib.smaug_get_state(eng.h, host_out.numpy().ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)), host_out.numel())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    te = torch.tensor([e2e_ms], device="cuda")
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * n_int * a.steps / (float(te.item()) / 1e3)
    state_bytes = host.numel() * 8
    h2d = state_bytes / a.steps
    d2h = state_bytes / a.steps + 8 * 8

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            cpu = cpu_throughput(nsteps=2)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # the GPU number stands on its own
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": max(3, a.warmup), "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"blast wave 3-D {a.n}^3 interior, periodic, RK4, hyperdiffusion on",
                       "ndim": 3, "interior": [a.n] * 3, "cells_with_ghosts": prob.ncells,
                       "parallelism": f"replicas x{world}", "l2": "state 4 x 8 fields x "
                       f"{prob.ncells} x 8 B = {4 * 8 * prob.ncells * 8 / 1e6:.0f} MB > 126 MB L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "stage_kernel<3>", "avg_launch_ms": avg_stage_ms,
                         "alg_bytes_per_launch": alg_bytes_per_launch},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
