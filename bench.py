"""Benchmark of the grand-potential explicit step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c4|c1] [--precision fp32|fp64]

One "step" is one explicit time step (phase-field half step, boundary copy,
concentration half step) of the whole workload, the unit of the reference's
time loop (microsim_gp.c:102-106).  The metric is cell-updates/s = interior
cells x steps / time.

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events on
the context's own stream, with an L2 flush (a 256 MiB write, more than the
126 MB L2) between timed steps and outside the events; the state of one 1024^2
instance would otherwise stay L2-resident.  Multi-GPU (torchrun): every rank
runs its own replica of the workload (the single-instance step does not
shard), barrier before and after, max over ranks.

The reference arm (--impl reference) times the reference serial solver,
compiled from its own sources (oracle/_ref/gp_ref_harness), on the host's
cores: one process per core, each on the same workload for a bounded number of
steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s (FP32 batched vs FP64 plain, 1 B200) at ≤0.5% tip-velocity err; % HBM"
UNIT = "cell-updates/s"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(name: str):
    from microsim_b200 import configs
    if name == "c2":
        return "dendrite_1024x1024_delta0.02_supersat0.55 (growing gap)", [configs.c2(literal=False, steps=50000)]
    if name == "c1":
        return "isotropic_200x200_seed10 (growing gap)", [configs.c1(literal=False, steps=10000)]
    if name == "c4":
        return "batched_sweep_256_instances_128-512", configs.c4()
    raise SystemExit("unknown workload " + name)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons while the timed region runs."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 4 + i and r[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return world, rank, local


def allmax(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------------------------- reference arm

def reference_rate(cases, steps: int, procs: int, timeout: float = 900.0):
    """Run the reference (compiled from source) on `procs` host cores, `steps` steps each.
    Returns (cell-updates/s aggregate, sample description)."""
    from oracle import gp_oracle as O
    if not os.path.exists(O.HARNESS_PATH):
        return None, "oracle/_ref/gp_ref_harness missing"
    case = max(cases, key=lambda c: c.cells)
    with tempfile.TemporaryDirectory() as td:
        case.write(td)
        ps = []
        for i in range(procs):
            wd = os.path.join(td, f"w{i}")
            os.makedirs(wd)
            for f in ("Input.in", "Filling.in"):
                os.link(os.path.join(td, f), os.path.join(wd, f))
            ps.append(subprocess.Popen([O.HARNESS_PATH, "Input.in", "Filling.in", "out", "-", str(steps)], cwd=wd,
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        secs = []
        for p in ps:
            out, _ = p.communicate(timeout=timeout)
            for line in out.splitlines():
                if line.startswith("loop_seconds="):
                    secs.append(float(line.split()[0].split("=")[1]))
    if len(secs) != procs:
        return None, "reference harness failed"
    rate = procs * case.cells * steps / max(secs)
    return rate, f"{case.mesh_x}x{case.mesh_y}, {steps} steps per process, {procs} processes (one per core)"


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    wname, cases = workload(args.workload)
    procs = max(1, min(os.cpu_count() or 1, 64))
    steps = max(1, args.ref_steps)
    t0 = time.time()
    rates = []
    sample = ""
    for _ in range(args.steps):
        r, sample = reference_rate(cases, steps, procs)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": sample}))
            return
        rates.append(r)
    v = statistics.median(rates)
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": wname, "sample_steps": steps, "processes": procs},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0}))


# --------------------------------------------------------------------------------------------- our arm

def run_ours(args, world, rank, local):
    import torch
    import microsim_b200 as mb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wname, cases = workload(args.workload)
    case = cases[0]
    prec = mb.GP_FP32 if args.precision == "fp32" else mb.GP_FP64
    with tempfile.TemporaryDirectory() as d:
        ip, fp = case.write(d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi0, mu0 = inp.fill(m)
    try:
        ctx = mb.Context(m, prec)
    except mb.GpError as e:
        if prec == mb.GP_FP32 and e.rc == mb.GP_E_UNSUPPORTED:
            prec = mb.GP_FP64
            args.precision = "fp64"
            ctx = mb.Context(m, prec)
        else:
            raise
    ctx.upload(phi0, mu0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    cells = m.mesh_x * m.mesh_y
    N, K1 = m.N, m.K1
    esize = 4 if prec == mb.GP_FP32 else 8
    alg_bytes = 2 * (N + K1) * esize  # read and write phi, mu once per cell-update

    for _ in range(args.warmup):
        ctx.step(1)
    ctx.sync()
    barrier(world)
    torch.cuda.synchronize()
    l0 = ctx.launches
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                evs[i][0].record(stream)
            ctx.step(1)
            with torch.cuda.stream(stream):
                evs[i][1].record(stream)
        ctx.sync()
    torch.cuda.synchronize()
    barrier(world)
    launches = ctx.launches - l0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    ms = allmax(ms, world)
    step_ms = ms / args.steps
    value = world * cells * args.steps / (ms / 1e3)
    per_gpu = cells / (step_ms / 1e3)
    peak, peak_kind = measured_peaks()
    achieved = per_gpu * alg_bytes / 1e9

    # end to end through the C ABI: pinned host state in, K steps with the
    # progress statistics read back each step, state out
    ph_t = torch.empty(phi0.shape, dtype=torch.float64, pin_memory=True)
    mu_t = torch.empty(mu0.shape, dtype=torch.float64, pin_memory=True)
    ph_h, mu_h = ph_t.numpy(), mu_t.numpy()
    ph_h[...] = phi0
    mu_h[...] = mu0
    ctx.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
    ctx.upload(ph_h, mu_h)
    for _ in range(args.steps):
        ctx.step(1)
        ctx.stats(allow_nonfinite=True)
    out_p, out_m = ctx.download()
    with torch.cuda.stream(stream):
        e1.record(stream)
    e1.synchronize()
    e2e_ms = allmax(e0.elapsed_time(e1), world)
    e2e = world * cells * args.steps / (e2e_ms / 1e3)
    state_bytes = (N + K1) * cells * 8
    stats_bytes = 64 * 8

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r, sample = reference_rate(cases, args.ref_steps, max(1, min(os.cpu_count() or 1, 64)))
        if r is not None:
            cpu = {"value": r, "unit": UNIT, "cores": max(1, min(os.cpu_count() or 1, 64)), "kind": "reference",
                   "sample": sample}
    ctx.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == mb.GP_FP32 else "f64", "data": "synthetic",
            "config": {"workload": wname, "precision": args.precision, "cells_per_gpu": cells,
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "flushed between timed steps (256 MiB write outside the events)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": f"algorithmic {alg_bytes} B/cell-update over the whole step; peak {peak_kind}"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps + stats_bytes},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c4"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--ref-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
