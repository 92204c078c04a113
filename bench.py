#!/usr/bin/env python3
"""Benchmark: ideal-MHD cell-updates/s on B200 (SAC/SMAUG method), batched
mixed precision against the plain FP64 single-simulation path.

Headline workload (one step = one full RK4 step of every simulation): the
batched ensemble of 96 independent 2-D Orszag-Tang vortices, sides drawn from
{128, 192, 256, 384, 512, 768} (seed 4242), B0 scaled by U[0.5, 1.5], 1 %
density noise, hyperdiffusion on, each with its own dt from the reference's
rule.  `value` is the batch (all 96 in one launch per RK stage, CUDA graphs,
mixed precision: FP32 stage states and stencils, FP64 backgrounds, pressure /
internal-energy recovery, RK base and sum, dt); "plain_fp64" times the same
96 simulations one after another through the FP64 single-simulation context.
The 3-D blast wave (128^3, FP64 and mixed, with an accuracy study against the
FP64 oracle build) is measured beside it ("blast128").
With --gpus N (torchrun) every rank advances its own replica (no data-path
collective: independent simulations), so scaling is weak.

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

METRIC = "cell-updates/s: batched mixed-prec vs plain FP64, 1 B200; p50/p99 latency"
UNIT = "cell-updates/s"
# Algorithmic HBM bytes per cell-update (one inner cell, one full RK4 step):
# the fused one-pass-per-stage minimum of SAC's fourstep, 14 evolved-field
# accesses (stage 1 reads U writes U1; 2 reads U1, U writes U2; 3 reads U2, U,
# U1 writes U3, U1'; 4 reads U3, U, U1' writes U) of NW fields plus 4 reads of
# the NB FP64 background fields: 14 NW s + 4 NB 8 bytes, s the state's element
# size (8 in FP64, 4 in the mixed path's FP32 states).
def alg_bytes_per_cell_update(ndim: int, mixed: bool) -> int:
    nw, nb = 2 + 2 * ndim, 2 + ndim
    return 14 * nw * (4 if mixed else 8) + 4 * nb * 8


BYTES_PER_CELL_UPDATE_FP64_2D = alg_bytes_per_cell_update(2, False)   # 800 B
BYTES_PER_CELL_UPDATE_MIXED_2D = alg_bytes_per_cell_update(2, True)   # 464 B
BYTES_PER_CELL_UPDATE_FP64_3D = alg_bytes_per_cell_update(3, False)   # 1056 B
BYTES_PER_CELL_UPDATE_MIXED_3D = alg_bytes_per_cell_update(3, True)   # 608 B
# What this design moves per cell-update in the mixed path (its traffic, not
# the algorithmic minimum): the RK base is an FP32 value plus an FP32
# compensation and the increment sum is an FP32 buffer, 19 FP32 field passes
# in all: 2-D 584 B, 3-D 768 B.
DESIGN_BYTES_MIXED = {2: 19 * 6 * 4 + 4 * 4 * 8, 3: 19 * 8 * 4 + 4 * 5 * 8}
ENSEMBLE = {"count": 96, "seed": 4242}
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
    """One simulation on one host core: (side, RK4-equivalent steps, timed
    seconds).  The reference's host code prints progress on stdout; it is sent
    to /dev/null so the bench's stdout keeps its one JSON line."""
    prob_args, substeps, min_steps, budget_s, use_ref = args
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    from smaug_b200 import problems
    prob = problems.orszag_tang(**prob_args)
    if use_ref:
        from oracle.oracle import Reference
        sim = Reference(prob)
        sim.step(1)  # warm-up: one reference single step
        adv = lambda: sim.step(substeps)  # noqa: E731
    else:
        from oracle.oracle import Oracle
        sim = Oracle(prob)
        sim.step(1, rk4=True)
        adv = lambda: sim.step(1, rk4=True)  # noqa: E731
    steps, t = 0, time.perf_counter()
    while steps < min_steps or (time.perf_counter() - t < budget_s and steps < 64):
        adv()
        steps += 1
    return prob_args["nx"], steps, time.perf_counter() - t


def _cpu_pool(jobs, procs):
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(_cpu_worker, jobs, chunksize=1)


def _use_ref() -> bool:
    return (ROOT / "oracle" / "_ref" / "libsmaug_ref2d.so").exists()


def cpu_throughput(procs: int | None = None, budget_s: float = 4.0):
    """Cell-updates/s of the reference's CPU code on the ensemble workload,
    from a bounded sample: one member of each side of the ensemble (128 ..
    768) advanced for at least one RK4-equivalent step (4 reference single
    steps; the reference's rkon=1 path is not usable) and for about
    `budget_s` seconds, one simulation per host process.  The per-side rates
    are combined with the 96-member ensemble's own mix of sides: time per
    ensemble step = sum over members of cells / rate(side), run on `procs`
    cores, so value = procs * cells / that time."""
    from smaug_b200 import problems
    use_ref = _use_ref()
    procs = procs or os.cpu_count() or 1
    substeps = SAMPLE_SUBSTEPS if use_ref else 1
    ens = problems.ensemble(ENSEMBLE["count"], seed=ENSEMBLE["seed"])
    sample = {}
    for i, p in enumerate(ens):  # the first member of each side
        side = p.n[0] - 4
        if side not in sample:
            m = p.meta
            sample[side] = dict(nx=side, b0_scale=m["b0_scale"], rho_noise=m["rho_noise"], seed=m["seed"])
    jobs = [(sample[s], substeps, 1, budget_s, use_ref) for s in sorted(sample, reverse=True)]
    t0 = time.perf_counter()
    res = _cpu_pool(jobs, min(procs, len(jobs)))
    wall = time.perf_counter() - t0
    rate = {side: side * side * steps / sec for side, steps, sec in res}  # cell-updates/s on one core
    cells = [p.interior for p in ens]
    t_one_core = sum(c / rate[int(round(c ** 0.5))] for c in cells)
    value = procs * sum(cells) / t_one_core
    kind = "reference" if use_ref else "port"
    desc = (f"one ensemble member of each side ({', '.join(str(s) for s in sorted(sample))}) for >= 1 RK4-equivalent "
            f"step and ~{budget_s:.0f} s each, one process per member"
            + (f" ({substeps} reference single steps per RK4-equivalent step; the reference's rkon=1 path is not "
               "usable)" if use_ref else " (oracle port, RK4)")
            + f"; per-side rates weighted by the 96-member mix, scaled to {procs} cores")
    return {"value": value, "unit": UNIT, "cores": procs, "kind": kind, "sample": desc,
            "per_side_rate_one_core": {str(k): v for k, v in sorted(rate.items())}, "wall_s": wall}


def cpu_c1(nsteps: int = 2):
    """The Orszag-Tang 256^2 workload on the host, through the reference's CPU
    build, `nsteps` RK4-equivalent steps, on 1 process and on nproc processes
    (one independent copy of the simulation per core: the reference's host
    build is single-threaded)."""
    use_ref = _use_ref()
    substeps = SAMPLE_SUBSTEPS if use_ref else 1
    args = dict(nx=256)
    nproc = os.cpu_count() or 1
    one = _cpu_pool([(args, substeps, nsteps, 0.0, use_ref)], 1)[0]
    many = _cpu_pool([(args, substeps, nsteps, 0.0, use_ref)] * nproc, nproc)
    cells = 256 * 256
    v1 = cells * one[1] / one[2]
    vn = sum(cells * r[1] for r in many) / max(r[2] for r in many)
    return {"kind": "reference" if use_ref else "port", "steps_timed": nsteps,
            "one_thread": {"value": v1, "unit": UNIT, "cores": 1,
                           "projected_1000_steps_s": 1000 * one[2] / one[1]},
            "nproc": {"value": vn, "unit": UNIT, "cores": nproc,
                      "note": "one independent copy per core (the reference's host build runs one simulation "
                              "on one thread)"}}


def run_reference(a):
    """The reference arm: the reference's CPU code on the host cores, on the
    same ensemble workload (a bounded sample, see cpu_throughput)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cpu = cpu_throughput()
    line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": dict(workload_config(a.gpus), precision="fp64 (the reference computes in FP64 only)",
                           same_config=True),
            "impl": "reference",
            "cpu_baseline": {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": cpu["kind"],
                             "sample": cpu["sample"]},
            "per_side_rate_one_core": cpu["per_side_rate_one_core"],
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def workload_config(world: int, cells: int | None = None, count: int = ENSEMBLE["count"]):
    return {"workload": f"batched ensemble: {count} independent 2-D Orszag-Tang vortices, sides {{128..768}} "
                        "(seed 4242), B0 x U[0.5,1.5], 1% density noise, periodic, RK4, hyperdiffusion on, "
                        "per-simulation dt (reference rule)",
            "ndim": 2, "simulations": count, "interior_cells": cells,
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2: ensemble state > 1 GB"}


# ----------------------------------------------------------------- GPU side

class ClockSampler:
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        # nvidia-smi numbers GPUs physically and ignores CUDA_VISIBLE_DEVICES:
        # select this process's device by its UUID
        self.uuid = None
        try:
            import torch
            u = str(torch.cuda.get_device_properties(device).uuid)
            self.uuid = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        self.proc = None
        # the raw samples (the line carries their summary): SMAUG_CLOCKS_DIR, else
        # the system's temporary directory
        import tempfile
        out = Path(os.environ.get("SMAUG_CLOCKS_DIR", tempfile.gettempdir()))
        self.path = out / f"smaug_clocks_rank{device}.csv"

    def start(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.f = open(self.path, "w")
            # line-buffered where stdbuf exists: no sample is lost in a buffer
            # when the sampler is stopped
            import shutil
            pre = ["stdbuf", "-oL"] if shutil.which("stdbuf") else []
            sel = self.uuid or str(self.device)
            self.proc = subprocess.Popen(pre + ["nvidia-smi", "-i", sel, f"--query-gpu={self.FIELDS}",
                                                "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, t_on: float | None = None, t_off: float | None = None):
        """Summary of the samples taken between host times t_on and t_off (one
        sampling period of slack each side; the first sample after t_on when
        none falls inside)."""
        import datetime
        if not self.proc:
            return None
        import signal
        self.proc.send_signal(signal.SIGINT)  # nvidia-smi ends its loop cleanly on SIGINT
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
            self.proc.wait()
        self.f.close()
        rows, later = [], []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                row = (float(parts[2]), float(parts[3]), parts[6:10])
            except ValueError:
                continue
            if t_on is None or t_on - 0.1 <= ts <= t_off + 0.1:
                rows.append(row)
            elif ts > t_on:
                later.append(row)
        rows = rows or later[:1]
        if not rows:
            return None
        sm = sorted(r[0] for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": rows[0][1], "reasons": reasons, "samples": len(rows),
                "gpu": self.uuid}


def event_ms(stream, fn):
    """Device time (ms) of the work fn() enqueues on `stream`."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


class Ctx:
    """Ranks, barrier and the max-over-ranks reduction of a time."""

    def __init__(self, a):
        import torch
        self.a = a
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(self.local)
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max_ms(self, ms: float) -> float:
        import torch
        t = torch.tensor([ms], device="cuda")
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def measure(eng, n_int, steps, warmup, ctx, sample_clocks):
    """Device-timed throughput of `steps` full steps of one engine, plus the
    average duration of its stage-kernel launches."""
    import torch
    stream = torch.cuda.ExternalStream(eng.stream)
    eng.step(max(3, warmup))
    eng.sync()
    sampler = ClockSampler(ctx.local) if sample_clocks else None
    if sampler:
        sampler.start()
    ctx.barrier()
    torch.cuda.synchronize()
    l0 = eng.launches
    ms = event_ms(stream, lambda: eng.step(steps))
    eng.sync()
    ctx.barrier()
    clocks = sampler.stop() if sampler else None
    launches = eng.launches - l0
    ms_max = ctx.max_ms(ms)
    eng.profile_stages(True)
    eng.step(max(2, min(steps, 8)))
    st_ms, st_n = eng.stage_times()
    eng.profile_stages(False)
    return {"value": ctx.world * n_int * steps / (ms_max / 1e3), "ms_per_step": ms_max / steps,
            "launches": launches, "clocks": clocks, "avg_stage_ms": st_ms / max(st_n, 1)}


def run_batched(probs, prec, ctx, steps, warmup, sample_clocks, force_variant=-1):
    """The whole ensemble in one batch: tune (or take force_variant), warm up,
    time `steps` steps."""
    import torch

    from smaug_b200 import Batch, footprint
    cells = sum(p.interior for p in probs)
    fp = sum(footprint(p, prec) for p in probs)
    b = Batch(2, precision=prec, arena_bytes=int(fp * 1.02) + (64 << 20), max_sims=len(probs), device=ctx.local)
    extra = 64  # steps beyond warm-up, timing and profiling: every simulation stays active throughout
    for p in probs:
        if b.add(p, warmup + steps + extra) is None:
            raise RuntimeError("ensemble does not fit its arena")
    # the clock sampler starts before the autotuner, so that it is sampling
    # when the timed region starts; only the samples inside that region count
    sampler = ClockSampler(ctx.local) if sample_clocks else None
    if sampler:
        sampler.start()
    variant, tune_ms = b.tune(reps=3)
    if force_variant >= 0:  # profiling one tile variant
        b.set_variant(force_variant)
        variant = force_variant
    stream = torch.cuda.ExternalStream(b.stream)
    b.step(warmup)
    b.sync()
    ctx.barrier()
    torch.cuda.synchronize()
    t_on = time.time()
    l0 = b.launches
    ms = event_ms(stream, lambda: b.step(steps))
    b.sync()
    t_off = time.time()
    ctx.barrier()
    clocks = sampler.stop(t_on, t_off) if sampler else None
    launches = b.launches - l0
    ms_max = ctx.max_ms(ms)
    b.profile_stages(True)
    b.step(2)
    st_ms, st_n = b.stage_times()
    b.profile_stages(False)
    b.close()
    return {"value": ctx.world * cells * steps / (ms_max / 1e3), "ms_per_step": ms_max / steps,
            "launches": launches, "clocks": clocks, "avg_stage_ms": st_ms / max(st_n, 1),
            "tile_variant": variant, "tune_stage1_ms": tune_ms}


def run_plain(probs, prec, ctx, steps, warmup):
    """The ensemble one simulation after another through the single-simulation
    context: the sum of their device times for `steps` steps each."""
    import torch

    from smaug_b200 import Engine
    cells = sum(p.interior for p in probs)
    tot = 0.0
    for p in probs:
        e = Engine(p, rk4=True, precision=prec, device=ctx.local)
        stream = torch.cuda.ExternalStream(e.stream)
        e.step(warmup)
        e.sync()
        tot += event_ms(stream, lambda: e.step(steps))
        e.sync()
        e.close()
    ms_max = ctx.max_ms(tot)
    return {"value": ctx.world * cells * steps / (ms_max / 1e3), "ms_per_step": ms_max / steps}


E2E_STEP_EVERY = 4  # admissions between the steps queued while the ensemble uploads (swept: 2, 4, 8, 16, 96)


def e2e_pipeline(b, probs, ws, mets, outs, steps: int):
    """Admit every simulation (state ws[i], metric mets[i]) into batch b,
    advance each by exactly `steps` steps (its budget at admission) and read
    each state into outs[i].  A step is queued every E2E_STEP_EVERY
    admissions, so the members admitted so far run while the next ones
    upload; the members admitted first then finish up to `queued` steps
    before the last one, and are read back (read-back stream, poll
    snapshots) while the last steps run."""
    slots, queued = [], 0
    for i, (p, w, m) in enumerate(zip(probs, ws, mets)):
        slots.append(b.add(p, steps, w=w, delx=m))
        if (i + 1) % E2E_STEP_EVERY == 0 and queued < steps:
            b.step(1)
            queued += 1
    pending = list(range(len(slots)))

    def read_finished(left):
        for k in [k for k in pending if left[slots[k]] == 0]:
            b.state_async(slots[k], outs[k])
            pending.remove(k)

    rest = steps
    first = rest - queued  # no member finishes before these are done
    if first:
        b.step(first)
    rest -= first
    tickets = [b.poll_begin()]
    while rest > 0:
        n = min(2, rest)
        b.step(n)
        rest -= n
        tickets.append(b.poll_begin())
        if len(tickets) > 2:  # the older snapshot: read what had finished there
            read_finished(b.poll_end(tickets.pop(0)))
    for tk in tickets:
        read_finished(b.poll_end(tk))
    b.io_wait()
    if pending:
        raise RuntimeError(f"e2e: {len(pending)} simulations did not finish their steps")
    return slots


def run_e2e_batched(probs, prec, ctx, steps):
    """End to end through the public batch API with host buffers: admit every
    simulation from pinned host memory, advance each by `steps` steps, read
    every result back into pinned host memory; uploads, steps and reads
    overlap as a serving loop overlaps them."""
    import numpy as np
    import torch

    from smaug_b200 import Batch, footprint
    cells = sum(p.interior for p in probs)
    fp = sum(footprint(p, prec) for p in probs)
    # host inputs, as a user holds them: each simulation's state and metric
    # in pinned memory
    ins = [torch.from_numpy(np.ascontiguousarray(p.w)).pin_memory() for p in probs]
    mets = [torch.from_numpy(np.concatenate([a.ravel() for a in p.delx()])).pin_memory() for p in probs]
    outs = [torch.empty_like(t).pin_memory() for t in ins]
    b = Batch(2, precision=prec, arena_bytes=int(fp * 1.02) + (64 << 20), max_sims=len(probs), device=ctx.local)
    stream = torch.cuda.ExternalStream(b.stream)
    ctx.barrier()
    torch.cuda.synchronize()

    def job():
        e2e_pipeline(b, probs, [t.numpy() for t in ins], [m.numpy() for m in mets], [o.numpy() for o in outs],
                     steps)

    ms = event_ms(stream, job)
    b.close()
    ms_max = ctx.max_ms(ms)
    nbytes = sum(t.numel() * 8 for t in ins)
    mbytes = sum(m.numel() * 8 for m in mets)  # admission copies the whole metric (checked on the device)
    return {"value": ctx.world * cells * steps / (ms_max / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": (nbytes + mbytes) / steps, "d2h_bytes_per_step": nbytes / steps}


def field_errors(w, ref, nw):
    """Per-field error over the inner cells: relative L2 ||x - y|| / ||y||; a
    field whose reference norm is zero or below 1e-9 of the largest field
    norm takes its absolute L2 over the largest field norm instead."""
    import numpy as np
    sl = (slice(0, nw),) + (slice(2, -2),) * (w.ndim - 1)
    x, y = w[sl], ref[sl]
    norms = np.array([np.linalg.norm(y[f]) for f in range(nw)])
    big = norms.max()
    return [float(np.linalg.norm(x[f] - y[f]) / (norms[f] if norms[f] > 1e-9 * big else big)) for f in range(nw)]


def accuracy_study(prob, steps: int, device: int, modes=("dt_rule", "fixed_dt"), dt_probe_steps: int | None = None,
                   checkpoints=()):
    """Per-field errors (field_errors) of the mixed and the FP64-FMA states
    against the FMA-free FP64 build (bit-identical to the oracle) after
    `steps` RK4 steps, under the reference's dt rule and at a fixed dt (half
    the dt the rule reaches after min(steps, dt_probe_steps) steps); the
    largest field error of both at each of `checkpoints` (steps) as well."""
    from smaug_b200 import PREC_MIXED, Engine

    nw = 2 + 2 * prob.ndim
    out = {"steps": steps, "reference": "FP64 FMA-free build (bit-identical to the oracle)"}
    probe = Engine(prob, rk4=True, device=device)
    probe.step(min(steps, dt_probe_steps or steps))
    dt_fixed = 0.5 * probe.scalars()["dt"]
    probe.close()
    for mode in modes:
        kw = {"dt_mode": 1} if mode == "dt_rule" else {"dt_mode": 0, "dt0": dt_fixed}
        ex = Engine(prob, rk4=True, exact=True, device=device, **kw)
        fa = Engine(prob, rk4=True, device=device, **kw)
        mi = Engine(prob, rk4=True, device=device, precision=PREC_MIXED, **kw)
        done, by_step = 0, []
        for n in [c for c in sorted(checkpoints) if 0 < c < steps]:
            for e in (ex, fa, mi):
                e.step(n - done)
            done = n
            w_n = ex.state()
            by_step.append({"step": n, "mixed_max_rel_l2": max(field_errors(mi.state(), w_n, nw)),
                            "fp64_fma_max_rel_l2": max(field_errors(fa.state(), w_n, nw))})
        for e in (ex, fa, mi):
            e.step(steps - done)
        we = ex.state()
        rm, rf = field_errors(mi.state(), we, nw), field_errors(fa.state(), we, nw)
        out[mode] = {"mixed_max_rel_l2": max(rm), "mixed_rel_l2_per_field": rm, "fp64_fma_max_rel_l2": max(rf),
                     "meets_1e-5": max(rm) <= 1e-5}
        if by_step:
            out[mode]["by_step"] = by_step
        if mode == "fixed_dt":
            out[mode]["dt"] = dt_fixed
        for e in (ex, fa, mi):
            e.close()
    return out


def run_c1(a, ctx):
    """The Orszag-Tang vortex 256^2, periodic, hyperdiffusion on,
    Courant 0.3, 1000 RK4 steps under the reference's dt rule, on the GPU
    through the single-simulation context (FP64 and mixed, CUDA events around
    the 1000 steps); the reference's CPU build on the same problem (a bounded
    sample at 1 thread and on every core); and the accuracy of 1000 steps,
    mixed and FP64-FMA against the FMA-free FP64 build, at a fixed dt and
    under the dt rule."""
    import torch

    from smaug_b200 import PREC_FP64, PREC_MIXED, Engine, problems
    prob = problems.orszag_tang(256)
    n_int = prob.interior
    out = {"workload": "Orszag-Tang 256^2 interior, periodic, gamma 5/3, hyperdiffusion on, Courant 0.3, "
                       "dt rule (moddton), RK4", "steps": a.c1_steps}
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        e = Engine(prob, rk4=True, precision=prec, device=ctx.local)
        e.step(max(3, a.warmup))
        e.sync()
        e.set_state(prob.w)  # the timed run starts from the initial state
        ms = ctx.max_ms(event_ms(torch.cuda.ExternalStream(e.stream), lambda: e.step(a.c1_steps)))
        e.sync()
        out[name] = {"value": ctx.world * n_int * a.c1_steps / (ms / 1e3), "unit": UNIT, "wall_ms": ms,
                     "final_dt": e.scalars()["dt"]}
        e.close()
    if ctx.rank == 0 and ctx.world == 1 and not a.no_cpu_baseline:
        try:
            out["cpu_reference"] = cpu_c1()
        except Exception as ex:  # the GPU numbers stand on their own
            out["cpu_reference"] = {"failed": str(ex)}
    if a.accuracy_steps > 0 and ctx.rank == 0:
        out["accuracy_1000_steps"] = accuracy_study(prob, a.c1_steps, ctx.local, dt_probe_steps=50,
                                                    checkpoints=(10, 30, 100, 300))
    return out


def run_blast(a, ctx):
    """3-D blast wave 128^3: mixed and FP64 single simulation, roofline of
    each, per-step host round trip end to end, accuracy study."""
    import ctypes

    import numpy as np
    import torch

    from smaug_b200 import PREC_FP64, PREC_MIXED, Engine, problems
    prob = problems.blast_wave(a.n, seed=1234 + ctx.rank)
    n_int = prob.interior
    peak, _ = load_peaks()
    out = {"workload": f"blast wave 3-D {a.n}^3 interior, periodic, RK4, hyperdiffusion on, single simulation",
           "cells_with_ghosts": prob.ncells}
    for name, prec, bpc in (("mixed", PREC_MIXED, BYTES_PER_CELL_UPDATE_MIXED_3D),
                            ("fp64", PREC_FP64, BYTES_PER_CELL_UPDATE_FP64_3D)):
        eng = Engine(prob, rk4=True, device=ctx.local, precision=prec)
        m = measure(eng, n_int, a.steps, a.warmup, ctx, sample_clocks=False)
        alg = bpc / 4 * n_int
        ach = alg / (m["avg_stage_ms"] / 1e3) / 1e9
        out[name] = {"value": m["value"], "ms_per_step": m["ms_per_step"], "avg_stage_ms": m["avg_stage_ms"],
                     "roofline": {"achieved": ach, "peak": peak, "frac": ach / peak, "unit": "GB/s",
                                  "alg_bytes_per_launch": alg}}
        if name == "mixed":
            out[name]["roofline"]["design_bytes_per_launch"] = DESIGN_BYTES_MIXED[3] / 4 * n_int
            # every step: smaug_set_state from pinned host memory, smaug_step,
            # smaug_get_state and smaug_get_scalars back to the host
            dptr = ctypes.POINTER(ctypes.c_double)
            host = torch.from_numpy(np.ascontiguousarray(prob.w)).pin_memory()
            hp = host.numpy().ctypes.data_as(dptr)
            scal = (ctypes.c_double * 8)()

            def loop():
                for _ in range(a.steps):
                    eng.lib.smaug_set_state(eng.h, hp, host.numel())
                    eng.lib.smaug_step(eng.h, 1)
                    eng.lib.smaug_get_state(eng.h, hp, host.numel())
                    eng.lib.smaug_get_scalars(eng.h, scal)

            ctx.barrier()
            torch.cuda.synchronize()
            ms = ctx.max_ms(event_ms(torch.cuda.ExternalStream(eng.stream), loop))
            out["mixed"]["e2e_per_step_round_trip"] = {
                "value": ctx.world * n_int * a.steps / (ms / 1e3), "h2d_bytes_per_step": host.numel() * 8,
                "d2h_bytes_per_step": host.numel() * 8 + 64}
        eng.close()
    out["mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    if a.accuracy_steps > 0 and ctx.rank == 0:
        out["accuracy"] = accuracy_study(prob, a.accuracy_steps, ctx.local)
        if a.c2_accuracy_steps > 0:  # the 128^3 blast wave: 500 steps at a fixed dt
            out["accuracy_500_steps_fixed_dt"] = accuracy_study(prob, a.c2_accuracy_steps, ctx.local,
                                                                modes=("fixed_dt",), dt_probe_steps=50,
                                                                checkpoints=(10, 50, 100, 250))
    return out


def run_atmos3d(a, ctx):
    """Stratified solar atmosphere, 3-D: 256 (z, vertical) x 128 x 128 cells over
    6 x 4 x 4 Mm; hydrostatic split background (T(z) tanh profile, rho_b by
    FP64 trapezoid from 2.7e-4 kg/m^3, uniform vertical B_b = 10 G); lower
    boundary vertical-velocity driver (300 s, 200 m/s, 0.5 Mm); vertical
    contcd4, lateral periodic; gravity.  Single simulation, mixed and FP64,
    then the mixed state's relative L2 difference from the FP64 one after the
    same steps."""
    import numpy as np

    from smaug_b200 import PREC_FP64, PREC_MIXED, Engine, problems
    prob = problems.atmosphere(256, 128, 128)
    n_int = prob.interior
    peak, _ = load_peaks()
    out = {"workload": "stratified atmosphere 3-D, 256 (z) x 128 x 128 cells over 6 x 4 x 4 Mm, hydrostatic "
                       "background, 10 G vertical B_b, lower-boundary driver 300 s / 200 m/s / 0.5 Mm, vertical "
                       "contcd4, lateral periodic, gravity, RK4, single simulation",
           "interior_cells": n_int}
    states = {}
    for name, prec, bpc in (("mixed", PREC_MIXED, BYTES_PER_CELL_UPDATE_MIXED_3D),
                            ("fp64", PREC_FP64, BYTES_PER_CELL_UPDATE_FP64_3D)):
        eng = Engine(prob, rk4=True, device=ctx.local, precision=prec)
        m = measure(eng, n_int, a.steps, a.warmup, ctx, sample_clocks=False)
        alg = bpc / 4 * n_int
        ach = alg / (m["avg_stage_ms"] / 1e3) / 1e9
        out[name] = {"value": m["value"], "ms_per_step": m["ms_per_step"], "avg_stage_ms": m["avg_stage_ms"],
                     "roofline": {"achieved": ach, "peak": peak, "frac": ach / peak, "unit": "GB/s",
                                  "alg_bytes_per_launch": alg}}
        states[name] = (eng.state(), eng.scalars()["steps"])
        eng.close()
    out["mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    wm, sm = states["mixed"]
    wf, sf = states["fp64"]
    nw = 2 + 2 * prob.ndim
    sl = (slice(None),) + tuple(slice(2, -2) for _ in range(prob.ndim))
    rel = []
    for f in range(nw):
        nb = float(np.linalg.norm(wf[sl][f]))
        rel.append(float(np.linalg.norm(wm[sl][f] - wf[sl][f]) / nb) if nb > 0 else None)
    out["mixed_vs_fp64_rel_l2_per_field"] = {"steps": sm, "same_steps": sm == sf, "fields": rel,
                                              "dt": "each path's own dt rule"}
    # the same comparison at one fixed dt: the dt rule's viscous limit comes
    # from hyperviscosity that the method computes from rounding noise in the
    # flat corona, so paths that round differently pick slightly different dt
    # and then drift apart; at a fixed dt what remains is the arithmetic
    dt0 = 0.1
    fixed = {}
    for name, prec in (("mixed", PREC_MIXED), ("fp64", PREC_FP64)):
        eng = Engine(prob, rk4=True, device=ctx.local, precision=prec, dt_mode=0, dt0=dt0)
        eng.step(20)
        fixed[name] = eng.state()
        eng.close()
    rel = []
    for f in range(nw):
        nb = float(np.linalg.norm(fixed["fp64"][sl][f]))
        rel.append(float(np.linalg.norm(fixed["mixed"][sl][f] - fixed["fp64"][sl][f]) / nb) if nb > 0 else None)
    out["mixed_vs_fp64_rel_l2_fixed_dt"] = {"steps": 20, "dt": dt0, "fields": rel}
    return out


def run_serving(a, ctx):
    """Serving stream: Poisson arrivals (40/s, seed 777) of driven
    stratified-atmosphere x-z slices, sizes {128x256 .. 512x1024}, driver
    period U[120,600] s, amplitude U[50,500] m/s, U[200,2000] steps, mixed
    precision, continuous batching; p50/p99 time to solution."""
    import torch

    from smaug_b200 import PREC_MIXED, Batch
    from smaug_b200.serve import Server, atmosphere_request_maker, merge_stats, poisson_stream, shard
    # one stream; with N GPUs each rank serves every N-th request as an
    # independent replica (its own batch, no data-path collective)
    stream = poisson_stream(a.serve_requests, 40.0, atmosphere_request_maker(), seed=777, duration=a.serve_seconds)
    reqs = shard(stream, ctx.rank, ctx.world)
    free, _ = torch.cuda.mem_get_info()
    arena = min(int(free * 0.5), 32 << 30)
    b = Batch(2, precision=PREC_MIXED, arena_bytes=arena, max_sims=256, device=ctx.local)
    ctx.barrier()
    srv = Server(b, chunk=10, keep_results=False, depth=2, time_chunks=True)
    st = srv.run(reqs, stop_after=a.serve_seconds)
    b.close()
    if ctx.dist is not None:  # the replicas' statistics, gathered once at the end
        gathered = [None] * ctx.world
        ctx.dist.all_gather_object(gathered, (st, srv.latencies))
        st = dict(st, **merge_stats(gathered))
    offered = sum(r.nsteps * r.prob.interior for r in stream)
    st.update({"arrival_rate_per_s": 40.0, "chunk_steps": 10, "pipeline_depth": 2, "arena_bytes": arena,
               "stream_seconds": a.serve_seconds,
               "offered_cell_updates_per_s": offered / max(stream[-1].arrival, 1e-9) if stream else 0.0,
               "replicas": ctx.world,
               "workload": f"Poisson arrivals 40/s (seed 777), {a.serve_requests} requests or {a.serve_seconds:.0f} s, "
                           "of driven atmosphere x-z slices {128x256, 256x512, 384x768, 512x1024}, period "
                           "U[120,600] s, amplitude U[50,500] m/s, U[200,2000] steps, mixed precision; the server "
                           "stops admitting and stepping at the stream's end; time to solution = arrival to result "
                           "on the host, over the requests completed by then"})
    return st


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128, help="blast wave: interior cells per dim")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 single-simulation ensemble run")
    ap.add_argument("--no-blast", action="store_true", help="skip the 3-D blast wave measurements")
    ap.add_argument("--no-atmos3d", action="store_true", help="skip the 3-D stratified atmosphere measurements")
    ap.add_argument("--only-batched", action="store_true", help="just the timed batched run (profiling)")
    ap.add_argument("--only-blast", action="store_true",
                    help="just the 3-D blast wave line, printed alone (profiling; --n sets its size)")
    ap.add_argument("--ensemble-count", type=int, default=ENSEMBLE["count"])
    ap.add_argument("--variant", type=int, default=-1,
                    help="tile variant of the batched mixed run (default: the autotuner's choice)")
    ap.add_argument("--serve-requests", type=int, default=2000, help="requests of the serving stream (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="length of the serving stream (s)")
    ap.add_argument("--accuracy-steps", type=int, default=50,
                    help="steps of the blast-wave accuracy study against the FP64 oracle build (0: skip all "
                         "accuracy studies)")
    ap.add_argument("--c1-steps", type=int, default=1000, help="RK4 steps of the Orszag-Tang 256^2 line (0: skip)")
    ap.add_argument("--c2-accuracy-steps", type=int, default=500,
                    help="steps of the blast-wave fixed-dt accuracy study (0: skip)")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference(a)

    from smaug_b200 import PREC_FP64, PREC_MIXED, problems
    ctx = Ctx(a)
    W, K = max(3, a.warmup), a.steps
    if a.only_blast:
        a.accuracy_steps = 0
        out = run_blast(a, ctx)
        if ctx.rank == 0:
            print(json.dumps({"blast": out}), flush=True)
        if ctx.dist is not None:
            ctx.barrier()
            ctx.dist.destroy_process_group()
        return 0
    probs = problems.ensemble(a.ensemble_count, seed=ENSEMBLE["seed"] + 1000 * ctx.rank)
    cells = sum(p.interior for p in probs)

    head = run_batched(probs, PREC_MIXED, ctx, K, W, sample_clocks=True, force_variant=a.variant)
    line_extra = {}
    if not a.only_batched:
        line_extra["batched_fp64"] = {k: v for k, v in run_batched(probs, PREC_FP64, ctx, K, W, False).items()
                                      if k in ("value", "ms_per_step", "avg_stage_ms", "tile_variant")}
        if not a.no_plain:
            plain = run_plain(probs, PREC_FP64, ctx, K, W)
            line_extra["plain_fp64"] = dict(plain, path="single-simulation context, FP64, one simulation after "
                                                        "another (smaug_create / smaug_step)")
            line_extra["batched_vs_plain_fp64"] = head["value"] / plain["value"]
        e2e = run_e2e_batched(probs, PREC_MIXED, ctx, K)
        if a.c1_steps > 0:
            line_extra["c1_ot256"] = run_c1(a, ctx)
        if not a.no_blast:
            line_extra["blast128"] = run_blast(a, ctx)
        if not a.no_atmos3d:
            line_extra["atmos3d"] = run_atmos3d(a, ctx)
        if a.serve_requests > 0:
            line_extra["serving"] = run_serving(a, ctx)
            sv = line_extra["serving"]
            # the served mix (driven atmosphere slices with live backgrounds) is
            # another workload than the headline ensemble: the device's own
            # throughput on that mix is the served cell-updates over the time
            # the GPU spent in chunks
            if sv.get("gpu_busy_s"):
                sv["device_cell_updates_per_s"] = sv["cell_updates"] / sv["gpu_busy_s"]
                sv["served_vs_device"] = sv["cell_updates_per_s"] / sv["device_cell_updates_per_s"]
            sv["served_vs_batched_headline"] = sv["cell_updates_per_s"] / head["value"]
    else:
        e2e = None

    alg = BYTES_PER_CELL_UPDATE_MIXED_2D / 4 * cells
    design = DESIGN_BYTES_MIXED[2] / 4 * cells
    achieved = alg / (head["avg_stage_ms"] / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    tr = load_traffic()
    kernel = "batch_stage_kernel<2,float>"
    # DRAM bytes per inner cell from the committed ncu capture, times this
    # run's inner cells (traffic grows with the cells a launch processes)
    per_cell = tr.get(kernel, {}).get("dram_bytes_per_inner_cell") if tr else None
    traffic = per_cell * cells if per_cell else None

    cpu = None
    if ctx.rank == 0 and ctx.world == 1 and not a.no_cpu_baseline and not a.only_batched:
        try:
            cpu = cpu_throughput()
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # the GPU number stands on its own
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}

    if ctx.rank == 0:
        cfg = workload_config(ctx.world, cells, a.ensemble_count)
        cfg["precision"] = "mixed: FP32 stage states/stencils; FP64 backgrounds, p_T, e_int, RK base + sum, dt"
        cfg["tile_variant"] = head["tile_variant"]
        # the autotuner's RK stage-1 time of every tile variant on this batch
        cfg["tile_variant_stage1_ms"] = [round(m, 4) for m in head["tune_stage1_ms"]]
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": ctx.world, "steps": K,
            "warmup": W, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": kernel, "avg_launch_ms": head["avg_stage_ms"], "alg_bytes_per_launch": alg,
                         "alg_bytes_basis": "464 B per cell-update / 4 stages (14 x 6 FP32 state + 4 x 4 FP64 "
                                            "background accesses per inner cell per RK4 step)",
                         "design_bytes_per_launch": design,
                         "design_frac": design / (head["avg_stage_ms"] / 1e3) / 1e9 / peak},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": head["launches"],
            "clocks": head["clocks"],
        }
        line.update(line_extra)
        print(json.dumps(line))
    if ctx.dist is not None:
        ctx.barrier()
        ctx.dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
