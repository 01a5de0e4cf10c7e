"""Benchmark of the grand-potential explicit step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c4|c2|c1]

One "step" is one explicit time step (phase-field half step, boundary copy,
concentration half step) of the whole workload, the unit of the reference's
time loop (microsim_gp.c:102-106).  The metric is cell-updates/s = interior
cells x steps / time.

Workloads: c4 (default) is the batched sweep the FP32-batched metric is quoted
on: 256 binary dendrite instances of sides 128..512, 25.1 M cells, one batch
(narrow band, CUDA-graph replay, autotuned tile); c2 a single 1024^2 dendrite;
c1 a single 200^2 seed.  The state is first advanced part-way through the run
(untimed), so the interfaces have grown.

Timing: W untimed warm-up steps, then K steps bracketed by CUDA events on the
batch's own stream.  A workload whose state fits in L2 is timed step by step
with an L2 flush (a 256 MiB write, more than the 126 MB L2) between steps and
outside the events; the batched sweep (301 MB per buffer) is larger than L2
and is timed as one graph-replayed run.  The same K steps are then replayed
with per-kernel CUDA events (direct launches) for the roofline of the dominant
kernel, and the FP64 plain step is timed on the same workload.  Multi-GPU
(torchrun): every rank runs its own batch of the sweep (distinct instances,
drawn from the rank's seed; a single-instance workload is replicated), no
data-path collective, barrier before and after, max over ranks of the time,
sum over ranks of the cells (microsim_b200/ranks.py).

The reference arm (--impl reference) times the reference serial solver,
compiled from its own sources (oracle/_ref/gp_ref_harness), on the host's
cores: one process per core, each on one instance of the workload (distinct
instances for the batched sweep) for a bounded number of steps, starting from
the same advanced state as the GPU arm (handed over as the reference's own
restart files; the CPU baseline of the GPU arm does the same).
"""
from __future__ import annotations

import argparse
import json
import os
import re
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
REF_BUDGET_S = 150.0  # wall-clock budget of the reference arm's samples
UNIT = "cell-updates/s"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(name: str, rank: int = 0, world: int = 1):
    from microsim_b200 import ranks
    return ranks.shard_workload(name, rank, world)


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
        import microsim_b200 as mb
        mb.set_device(local)  # the library's own CUDA runtime
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return world, rank, local


def allmax(v: float, world: int) -> float:
    from microsim_b200 import ranks
    return ranks.allreduce(v, world, "max")


def allsum(v: float, world: int) -> float:
    from microsim_b200 import ranks
    return ranks.allreduce(v, world, "sum")


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------------------------- reference arm

def reference_rate(cases, steps: int, procs: int, timeout: float = 900.0, start=None):
    """Run the reference (compiled from source) on `procs` host cores, `steps` steps each.
    With start = (t, fields): every process starts from its instance's state after t steps
    (fields[i] = (phi, mu)), handed to the reference as its own restart file (DATA/out_<t>.vtk in
    the input's WRITEFORMAT, read by its RESTART path), so it times the same workload state as
    the GPU arm.  Returns (cell-updates/s aggregate, sample description)."""
    from oracle import gp_oracle as O
    if not os.path.exists(O.HARNESS_PATH):
        return None, "oracle/_ref/gp_ref_harness missing"
    # one instance per process: the workload's instances in turn (a single-instance workload repeats it)
    idx = [i % len(cases) for i in range(procs)]
    chosen = [cases[i] for i in idx]
    with tempfile.TemporaryDirectory() as td:
        ps = []
        for i, case in enumerate(chosen):
            wd = os.path.join(td, f"w{i}")
            os.makedirs(wd)
            ip, fp = case.write(wd)
            if start is not None:
                import microsim_b200 as mb
                t0, fields = start
                text = open(ip).read()
                text = re.sub(r"(?m)^STARTTIME\s*=\s*\d+;", f"STARTTIME = {t0};", text)
                text = re.sub(r"(?m)^RESTART\s*=\s*\d+;", "RESTART = 1;", text)
                open(ip, "w").write(text)
                os.makedirs(os.path.join(wd, "DATA"), exist_ok=True)
                inp = mb.Input(ip, fp)
                inp.write_vtk(inp.model(), os.path.join(wd, "DATA", f"out_{t0}.vtk"), *fields[idx[i]], t0)
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
    rate = sum(c.cells for c in chosen) * steps / max(secs)
    sides = sorted({f"{c.mesh_x}x{c.mesh_y}" for c in chosen})
    state = (f"from the state after {start[0]} steps (the GPU arm's, as the reference's restart file)"
             if start is not None else "from the initial filling")
    return rate, (f"{procs} processes (one per core), one instance each ({', '.join(sides)}), "
                  f"{steps} steps per process {state}; rate = cells x steps / slowest process")


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    wname, cases = workload(args.workload)
    procs = max(1, min(os.cpu_count() or 1, 64))
    steps = max(1, args.ref_steps)
    t0 = time.time()
    # input preparation, outside every timed region: the workload state the GPU arm times (its
    # instances advanced by the FP32 form), handed to the reference as its own restart files; the
    # timed runs are the reference alone
    start = None
    prep = args.prep_steps if args.prep_steps >= 0 else {"c2": 25000, "c1": 5000, "c4": 2500}[args.workload]
    try:
        import microsim_b200 as mb
        loaded = [mb.load_case(c) for c in cases[:procs]]
        start = (prep, prepare([m for m, _, _ in loaded], [(p, u) for _, p, u in loaded], prep))
    except Exception:  # no GPU or library: the reference starts from the initial filling (said in `sample`)
        start = None
    rates = []
    sample = ""
    # K samples, each a bounded run of the reference; the whole arm stays within a few minutes:
    # after three samples, no new one starts once REF_BUDGET_S have passed (the line says how many ran)
    t_run = time.time()
    for _ in range(args.steps):
        if len(rates) >= 3 and time.time() - t_run > REF_BUDGET_S:
            break
        r, sample = reference_rate(cases, steps, procs, start=start)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": sample}))
            return
        rates.append(r)
    v = statistics.median(rates)
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": wname, "sample_steps": steps, "processes": procs,
                                        "samples_run": len(rates), "value_is": "median over the samples"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0}))


# --------------------------------------------------------------------------------------------- our arm

def prepare(models, fields, steps, compensated=False):
    """Advance the synthetic initial state `steps` steps with the FP32 form (input
    preparation, before any timing): the benchmark state is the workload part-way
    through its run, where the interface has grown, instead of the first steps of a
    small seed."""
    import microsim_b200 as mb
    if steps <= 0:
        return fields
    with mb.Batch(models) as b:
        b.set_compensated(compensated)
        for i, (p, u) in enumerate(fields):
            b.upload(i, p, u)
        b.step(steps)
        b.sync()
        return [b.download(i) for i in range(len(models))]


def timed_single(ctx, steps, warmup, flush, stream):
    """Per-step CUDA events on the context's stream, L2 flushed between steps."""
    import torch
    for _ in range(warmup):
        ctx.step(1)
    ctx.sync()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    l0 = ctx.launches
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches
    for i in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            evs[i][0].record(stream)
        ctx.step(1)
        with torch.cuda.stream(stream):
            evs[i][1].record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    return sum(a.elapsed_time(b) for a, b in evs), ctx.launches - l0


def traffic_table():
    """Per-launch DRAM bytes of the step kernels measured by ncu on the bench
    workloads (profiles/dram_traffic.txt: "<workload> <kernel> <bytes>")."""
    t = {}
    p = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if os.path.exists(p):
        for line in open(p):
            f = line.split()
            if len(f) == 3 and not line.startswith("#"):
                t[(f[0], f[1])] = float(f[2])
    return t


def fp64_plain_rate(models, fields, steps, warmup, dev, world):
    """FP64 plain step (bit-exact to the reference) over every instance of the
    workload: one context per instance, each on its own stream, all stepped
    concurrently; K steps between a CUDA event on a master stream (which every
    context's stream waits on) and the master's wait on every context's end
    event.  An isothermal context replays its steps from a CUDA graph (gp_step),
    captured during the warm-up."""
    import torch
    import microsim_b200 as mb
    ctxs = []
    try:
        for m, (p, u) in zip(models, fields):
            c = mb.Context(m, mb.GP_FP64)
            ctxs.append(c)
            c.upload(p, u)
            c.step(warmup)
        for c in ctxs:
            c.sync()
        torch.cuda.synchronize()
        master = torch.cuda.Stream(device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(master)
        streams = [torch.cuda.ExternalStream(c.stream, device=dev) for c in ctxs]
        for s in streams:
            s.wait_event(e0)
        for c in ctxs:
            c.step(steps)
        for s in streams:
            ev = torch.cuda.Event()
            ev.record(s)
            master.wait_event(ev)
        e1.record(master)
        e1.synchronize()
        total_ms = e0.elapsed_time(e1)
        cells = sum(m.mesh_x * m.mesh_y for m in models)
    finally:
        for c in ctxs:
            c.close()
    total_ms = allmax(total_ms, world)
    return {"value": allsum(cells, world) * steps / (total_ms / 1e3), "unit": UNIT, "ms_per_step": total_ms / steps,
            "how": f"{len(models)} contexts, one stream each, stepped concurrently"}


def run_ours(args, world, rank, local):
    import torch
    import microsim_b200 as mb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wname, cases = workload(args.workload, rank, world)
    loaded = [mb.load_case(c) for c in cases]
    models = [m for m, _, _ in loaded]
    prep = args.prep_steps if args.prep_steps >= 0 else {"c2": 25000, "c1": 5000, "c4": 2500}[args.workload]
    comp = args.compensated == 1
    fields = prepare(models, [(p, u) for _, p, u in loaded], prep, comp)
    cells = sum(m.mesh_x * m.mesh_y for m in models)
    N, K1 = models[0].N, models[0].K1
    peak, peak_kind = measured_peaks()
    barrier(world)

    # ---- the chosen form (FP32 batch: narrow band, CUDA-graph replay)
    ctx = mb.Batch(models)
    ctx.set_compensated(comp)
    for i, f in enumerate(fields):
        ctx.upload(i, *f)
    tile = ctx.autotune(args.tune_cache) if not args.no_autotune else (16, 32)
    ctx.prepare()  # graph capture is set-up, not part of a step
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    state_mb = cells * (N + K1) * 4 / 1e6
    with ClockSampler(local) as clk:
        if state_mb < 300:  # would stay L2-resident: flush between steps, per-step events
            flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
            ms, launches = timed_single(ctx, args.steps, args.warmup, flush, stream)
            l2 = "flushed between timed steps (256 MiB write outside the events)"
        else:
            ctx.step(args.warmup)
            ctx.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = ctx.launches
            torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches
            with torch.cuda.stream(stream):
                e0.record(stream)
            ctx.step(args.steps)
            with torch.cuda.stream(stream):
                e1.record(stream)
            ctx.sync()
            torch.cuda.nvtx.range_pop()
            launches = ctx.launches - l0
            ms = e0.elapsed_time(e1)
            l2 = "inputs larger than L2 (state %.0f MB per buffer)" % state_mb
    torch.cuda.synchronize()
    barrier(world)
    ms = allmax(ms, world)
    step_ms = ms / args.steps
    cells_all = allsum(cells, world)  # every rank's own instances
    value = cells_all * args.steps / (ms / 1e3)

    # ---- per-kernel CUDA-event timing of the same steps (direct launches)
    lean_tiles, tiles, lean_cells = ctx.lean_stats()
    ctx.set_timing(True)
    ctx.step(args.steps)
    kt = ctx.kernel_ms()
    ctx.set_timing(False)
    gen_cells = cells - lean_cells
    depth = ctx.depth()
    grids = ctx.grids()
    if depth == 2:  # per blocked pair (two steps): kernel_ms reports per step
        kernels = {
            "k_lean2": {"ms": 2 * kt["lean"], "bytes": 2 * lean_cells * 2 * K1 * 4,
                        "what": f"mu read + write of the {lean_tiles} lean tiles for each of the pair's two steps "
                                f"({2 * K1 * 4} B/cell/step; the pair itself moves mu once, read at t and written "
                                f"at t+2); launches of the pair: adjacency list, lean tiles next to the interface "
                                f"tiles, the other lean tiles"},
            "k_step32": {"ms": 2 * kt["general"], "bytes": 2 * gen_cells * 2 * (N + K1) * 4,
                         "what": f"phi, mu read + write of the {tiles - lean_tiles} other tiles, two passes "
                                 f"({2 * (N + K1) * 4} B/cell/step)"},
            "k_general_list": {"ms": 2 * kt["list"], "bytes": tiles * 4 * 9, "what": "purity words"},
        }
    else:
        kernels = {
            "k_lean32": {"ms": kt["lean"], "bytes": lean_cells * 2 * K1 * 4,
                         "what": f"mu read + write of the {lean_tiles} lean tiles ({2 * K1 * 4} B/cell)"},
            "k_step32": {"ms": kt["general"], "bytes": gen_cells * 2 * (N + K1) * 4,
                         "what": f"phi, mu read + write of the {tiles - lean_tiles} other tiles "
                                 f"({2 * (N + K1) * 4} B/cell)"},
            "k_general_list": {"ms": kt["list"], "bytes": tiles * 4 * 9, "what": "purity words"},
        }
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    d = kernels[dom]
    achieved = d["bytes"] / (d["ms"] / 1e3) / 1e9 if d["ms"] > 0 else None
    traffic = traffic_table().get((args.workload, dom))
    esize = 4
    alg_bytes = 2 * (N + K1) * esize

    # ---- dense FP32 (narrow band off: every tile through the full kernel, phi and mu moved every
    # step): the chosen form's precision and kernels without the narrow band or temporal blocking
    dense = None
    if not args.no_fp64:
        nb_depth = ctx.depth()
        ctx.set_narrowband(False)
        ctx.prepare()
        ctx.step(args.warmup)
        ctx.sync()
        ed0, ed1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ed0.record(stream)
        ctx.step(args.steps)
        with torch.cuda.stream(stream):
            ed1.record(stream)
        ctx.sync()
        dms = allmax(ed0.elapsed_time(ed1), world)
        dval = cells_all * args.steps / (dms / 1e3)
        dach = dval / world * alg_bytes / 1e9
        dense = {"value": dval, "unit": UNIT, "ms_per_step": dms / args.steps,
                 "roofline": {"bound": "hbm", "achieved": dach, "peak": peak, "unit": "GB/s", "frac": dach / peak,
                              "alg_bytes_per_cell": alg_bytes,
                              "note": "phi and mu read + write once per cell-update, every tile"}}
        ctx.set_narrowband(True)
        ctx.set_depth(nb_depth)

    # ---- the other FP32 accumulation mode on the same configuration (its cost per step)
    other = None
    if not args.no_fp64:
        ctx.set_compensated(not comp)
        ctx.prepare()
        ctx.step(args.warmup)
        ctx.sync()
        eo0, eo1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            eo0.record(stream)
        ctx.step(args.steps)
        with torch.cuda.stream(stream):
            eo1.record(stream)
        ctx.sync()
        oms = allmax(eo0.elapsed_time(eo1), world)
        other = {"accumulation": "plain" if comp else "compensated (TwoSum/TwoProduct)",
                 "value": cells_all * args.steps / (oms / 1e3), "unit": UNIT, "ms_per_step": oms / args.steps,
                 "note": "same tiles, grids and depth as the headline; graphs recaptured for this mode"}
        ctx.set_compensated(comp)

    # ---- FP64 plain on the same workload
    fp64 = None
    if not args.no_fp64:
        # as many warm-up steps as timed ones: the timed steps then take the launch path (graph
        # replays of isothermal runs, direct launches of the rest) that the warm-up prepared
        fp64 = fp64_plain_rate(models, fields, 16, 16, dev, world)

    # ---- end to end through the C ABI: pinned host state in, K steps with the
    # progress statistics read back each step, state out
    pinned = []
    for p, u in fields:
        pt = torch.empty(p.shape, dtype=torch.float64, pin_memory=True)
        ut = torch.empty(u.shape, dtype=torch.float64, pin_memory=True)
        pt.numpy()[...] = p
        ut.numpy()[...] = u
        pinned.append((pt.numpy(), ut.numpy()))
    pinned_out = [(torch.empty(p.shape, dtype=torch.float64, pin_memory=True).numpy(),
                   torch.empty(u.shape, dtype=torch.float64, pin_memory=True).numpy()) for p, u in fields]
    raw = torch.zeros((args.steps, mb.GP_STAT_VALUES), dtype=torch.float64, pin_memory=True).numpy()
    # one untimed round trip through the same page-locked buffers first (warm-up: the first
    # transfer from freshly page-locked memory runs at about half the link's speed)
    ctx.upload_all(pinned)
    ctx.download_all(pinned_out)
    ctx.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
    ctx.upload_all(pinned)  # every instance in one queued conversion launch reading the host arrays
    for t in range(args.steps):
        ctx.step(1)
        ctx.stats_async(0, raw[t])  # the step's result read back to the host, queued (no wait per step)
    ctx.download_all(pinned_out)
    with torch.cuda.stream(stream):
        e1.record(stream)
    e1.synchronize()
    ctx.sync()
    e2e_ms = allmax(e0.elapsed_time(e1), world)
    for t in range(args.steps):  # every step's statistics arrived (decoded outside the timed region)
        if not np.isfinite(ctx.stats_from_raw(0, raw[t], allow_nonfinite=True)["solute"][0]):
            raise RuntimeError(f"non-finite solute after end-to-end step {t + 1}")
    e2e = cells_all * args.steps / (e2e_ms / 1e3)
    state_bytes = (N + K1) * cells * 8

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = max(1, min(os.cpu_count() or 1, 64))
        r, sample = reference_rate(cases, args.ref_steps, procs, start=(prep, fields))
        if r is not None:
            cpu = {"value": r, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample}
    ctx.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wname, "precision": "fp32", "instances": len(models), "cells_per_gpu": cells,
                       "state_prepared_steps": prep,
                       "parallelism": (f"instances sharded over {world} ranks" if len(models) > 1 else
                                       f"replicas{world}") if world > 1 else "single", "l2": l2,
                       "tile": list(tile), "lean_tiles": lean_tiles, "tiles": tiles, "depth": depth,
                       "blocks_per_sm": {"lean": grids[0], "full": grids[1]},
                       "accumulation": "compensated (TwoSum/TwoProduct)" if comp else "plain"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": traffic,
                         "bytes_per_launch": d["bytes"], "ms_per_launch": d["ms"],
                         "note": f"dominant kernel {dom}: algorithmic bytes = {d['what']} / its mean CUDA-event "
                                 f"duration; peak {peak_kind}; traffic = ncu dram bytes per launch "
                                 f"(profiles/dram_traffic.txt); temporal blocking depth {depth}"},
            "step_roofline": {"alg_bytes_per_cell": alg_bytes, "achieved": value / world * alg_bytes / 1e9,
                              "frac": value / world * alg_bytes / 1e9 / peak,
                              "note": "dense-step definition: read+write phi and mu once per cell-update; the "
                                      "narrow band skips phi traffic of pure tiles, so this can exceed 1"},
            # a blocked pair's launches cover two steps: per step is half of it
            "kernels_ms_per_step": {k: v["ms"] / depth for k, v in kernels.items()},
            ("fp32_compensated" if not comp else "fp32_plain_accumulation"): other,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps + 64 * 8},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if depth == 2:
            line["kernels_ms_per_pair"] = {k: v["ms"] for k, v in kernels.items()}
        if dense:
            line["fp32_dense"] = dense
        if fp64:
            alg64 = 2 * (N + K1) * 8
            fp64["roofline"] = {"bound": "hbm", "achieved": fp64["value"] / world * alg64 / 1e9, "peak": peak,
                                "unit": "GB/s", "frac": fp64["value"] / world * alg64 / 1e9 / peak,
                                "alg_bytes_per_cell": alg64}
            line["fp64_plain"] = fp64
            line["fp32_over_fp64"] = value / fp64["value"]
            if dense:  # the speed-up in parts: precision and kernels, then narrow band and blocking
                line["speedup_parts"] = {"fp32_dense_over_fp64": dense["value"] / fp64["value"],
                                         "narrowband_and_blocking_over_dense": value / dense["value"]}
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c1", "c2", "c4"])
    ap.add_argument("--ref-steps", type=int, default=50)
    ap.add_argument("--prep-steps", type=int, default=-1,
                    help="steps of the FP32 form run before timing to reach a mid-run state (-1: half the run)")
    ap.add_argument("--compensated", type=int, default=0, choices=[0, 1],
                    help="FP32 accumulation of the headline: plain (0, default) or compensated (1); the other "
                         "mode is timed on the same configuration beside it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner cache file: a profiled rerun reads back the plain run's choice")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        # rank 0 alone runs the reference on the host cores; the other ranks exit without work
        # (no process group: nothing in this arm is collective)
        rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
        if rank == 0:
            run_reference_arm(args, world, rank)
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
