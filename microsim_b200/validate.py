"""FP32 chosen form against the FP64 plain form, per workload.

    python -m microsim_b200.validate [--workload c2|c4|c1|c3] [--steps S] [--every E] [--mesh M]
                                     [--compensated 0|1|both]

Runs each instance of the workload in both forms (the FP32 form through the
batch API, narrow band on; the FP64 plain form one context per instance),
samples every `every` steps the tip position along the growth axis through the
seed (phi_solid = 0.5 crossing), the tip radius (corner dendrites), the FP64
solute mass and the phase fractions, and prints the relative differences of
the FP32 form:
  * tip velocity: least-squares slope of the tip position over the last fifth
    of the run (restating resources/PP_tools/frontvelocity.py);
  * final tip position and radius (resources/PP_tools/tipradius.py);
  * solute mass and phase fractions at the end, and each form's solute drift
    (relative change of the solute mass from the first sample to the last).
The FP32 form runs with plain or compensated accumulation (--compensated), or
both against one FP64 run.
Workloads: c2 the 1024^2 corner dendrite (50,000 steps), c4 the 256-instance
batched sweep (5,000 steps), c1 the 200^2 centred seed (10,000 steps), c3 the
2048^2 four-phase ternary (20,000 steps; no single tip: phase fractions and
solute mass only).  The growing-gap variants of the configs are used
(microsim_b200/configs.py).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import GP_FP32, GP_FP64, Batch, Context, analysis as A, configs, load_case


def _sample(m, p, st, line):
    tip = A.tip_position(p[0], 0, line)
    rad = A.tip_radius(p[0], 0) if line == 0 else float("nan")
    fr = [float(p[a].mean()) for a in range(m.N)]
    return [tip, rad, *st["solute"][: m.K1], *fr, st["nonfinite"]]


def run_fp32(models, loaded, lines, steps, every, compensated=False):
    rec = [[] for _ in models]
    with Batch(models) as b:
        b.set_compensated(compensated)
        for i, (_, p, u) in enumerate(loaded):
            b.upload(i, p, u)
        for s in range(every, steps + 1, every):
            b.step(every)
            for i, m in enumerate(models):
                p, _ = b.download(i)
                rec[i].append([s, *_sample(m, p, b.stats(i, allow_nonfinite=True), lines[i])])
    return [np.array(r) for r in rec]


def run_fp64(models, loaded, lines, steps, every):
    out = []
    for (m, phi, mu), line in zip(loaded, lines):
        rec = []
        with Context(m, GP_FP64) as c:
            c.upload(phi, mu)
            for s in range(every, steps + 1, every):
                c.step(every)
                p, _ = c.download()
                rec.append([s, *_sample(m, p, c.stats(allow_nonfinite=True), line)])
        out.append(np.array(rec))
    return out


def _rel(a, b):
    return float(abs(a - b) / abs(b)) if b != 0 else float(abs(a - b))


def _differences(workload, models, f32, f64):
    per = []
    for m, a, b in zip(models, f32, f64):
        K1, N = m.K1, m.N
        w = max(3, len(b) // 5)
        r = {"solute_rel_diff": max(_rel(a[-1, 3 + k], b[-1, 3 + k]) for k in range(K1)),
             "solute_drift_fp32": max(_rel(a[-1, 3 + k], a[0, 3 + k]) for k in range(K1)),
             "solute_drift_fp64": max(_rel(b[-1, 3 + k], b[0, 3 + k]) for k in range(K1)),
             "phase_fraction_abs_diff": float(np.abs(a[-1, 3 + K1:3 + K1 + N] - b[-1, 3 + K1:3 + K1 + N]).max()),
             "nonfinite": int(a[:, -1].max() + b[:, -1].max())}
        if workload != "c3":
            v64 = A.velocity(b[:, 0] * m.dt, b[:, 1], w)
            v32 = A.velocity(a[:, 0] * m.dt, a[:, 1], w)
            r.update({"tip_velocity_fp64": v64, "tip_velocity_fp32": v32, "tip_velocity_rel_err": _rel(v32, v64),
                      "tip_position_rel_err": _rel(a[-1, 1], b[-1, 1])})
            if not np.isnan(b[-1, 2]):
                r["tip_radius_rel_err"] = _rel(a[-1, 2], b[-1, 2])
        per.append(r)
    out = {}
    keys = sorted({k for r in per for k in r})
    for k in keys:
        vals = [r[k] for r in per if k in r and not (isinstance(r[k], float) and np.isnan(r[k]))]
        if not vals:
            continue
        if len(per) == 1:
            out[k] = vals[0]
        else:
            out[k + "_max"] = max(vals)
            out[k + "_median"] = float(np.median(vals))
    return out


def compare(workload: str = "c2", steps: int | None = None, every: int | None = None, mesh: int | None = None,
            instances: int | None = None, compensated=(False,)) -> dict:
    """FP32 (each accumulation mode in `compensated`) against one FP64 run; with
    one mode the differences are top-level keys, with several they sit under
    "plain" and "compensated"."""
    t0 = time.time()
    if workload == "c2":
        steps, every = steps or 50000, every or 1000
        cases = [configs.c2(literal=False, steps=steps, mesh=mesh or 1024)]
    elif workload == "c4":
        steps, every = steps or 5000, every or 250
        cases = configs.c4(steps=steps)[: instances or 256]
    elif workload == "c1":
        steps, every = steps or 10000, every or 500
        cases = [configs.c1(literal=False, steps=steps)]
    elif workload == "c3":
        steps, every = steps or 20000, every or 1000
        cases = [configs.c3(steps=steps, mesh=mesh or 2048)]
    else:
        raise ValueError(workload)
    loaded = [load_case(c) for c in cases]
    models = [m for m, _, _ in loaded]
    lines = [0 if (c.fills[0][1][1] == 0 and c.fills[0][1][2] == 0) else int(c.fills[0][1][2]) for c in cases]
    f32 = {c: run_fp32(models, loaded, lines, steps, every, c) for c in compensated}
    f64 = run_fp64(models, loaded, lines, steps, every)
    out = {"workload": workload, "instances": len(models), "steps": steps, "every": every}
    if len(models) == 1:
        m = models[0]
        out["phase_fraction_fp64"] = [float(v) for v in f64[0][-1, 3 + m.K1:3 + m.K1 + m.N]]
        out["phase_fraction_fp64_start"] = [float(v) for v in f64[0][0, 3 + m.K1:3 + m.K1 + m.N]]
    if len(compensated) == 1:
        out["compensated"] = bool(compensated[0])
        out.update(_differences(workload, models, f32[compensated[0]], f64))
    else:
        for c in compensated:
            out["compensated" if c else "plain"] = _differences(workload, models, f32[c], f64)
    out["wall_s"] = time.time() - t0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2", choices=["c2", "c4", "c1", "c3"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--every", type=int, default=None)
    ap.add_argument("--mesh", type=int, default=None)
    ap.add_argument("--instances", type=int, default=None)
    ap.add_argument("--compensated", default="0", choices=["0", "1", "both"],
                    help="FP32 accumulation: plain (0), compensated (1) or both against one FP64 run")
    a = ap.parse_args()
    modes = (False, True) if a.compensated == "both" else (a.compensated == "1",)
    print(json.dumps(compare(a.workload, a.steps, a.every, a.mesh, a.instances, modes)))


if __name__ == "__main__":
    main()
