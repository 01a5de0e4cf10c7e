"""FP32 chosen form against the FP64 plain form on one workload.

    python -m microsim_b200.validate [--mesh 1024] [--steps 50000] [--every 1000]

Runs the corner dendrite of the 1024^2 workload (4-fold, delta = 0.02,
supersaturation 0.55, growing-gap variant) in both forms, samples the tip
position, tip radius, solute mass and solid fraction every `every` steps, and
prints the relative errors of the FP32 form: tip velocity (least-squares slope
over the last fifth of the run), final tip position and radius, solute mass.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import GP_FP32, GP_FP64, Context, analysis as A, configs, load_case


def run(mesh: int = 1024, steps: int = 50000, every: int = 1000, precision: int = GP_FP64):
    case = configs.c2(literal=False, steps=steps, mesh=mesh)
    m, phi, mu = load_case(case)
    rec = []
    with Context(m, precision) as c:
        c.upload(phi, mu)
        for s in range(every, steps + 1, every):
            c.step(every)
            p, _ = c.download()
            st = c.stats(allow_nonfinite=True)
            rec.append([s, A.tip_position(p[0], 0), A.tip_position(p[0], 1), A.tip_radius(p[0], 0),
                        st["solute"][0], A.solid_fraction(p), st["nonfinite"]])
    return m, np.array(rec)


def compare(mesh: int = 1024, steps: int = 50000, every: int = 1000) -> dict:
    t0 = time.time()
    m, f32 = run(mesh, steps, every, GP_FP32)
    _, f64 = run(mesh, steps, every, GP_FP64)
    w = max(3, len(f64) // 5)
    v64 = A.velocity(f64[:, 0] * m.dt, f64[:, 1], w)
    v32 = A.velocity(f32[:, 0] * m.dt, f32[:, 1], w)
    return {
        "mesh": mesh, "steps": steps, "every": every,
        "tip_velocity_fp64": v64, "tip_velocity_fp32": v32,
        "tip_velocity_rel_err": abs(v32 - v64) / abs(v64),
        "tip_position_rel_err": abs(f32[-1, 1] - f64[-1, 1]) / f64[-1, 1],
        "tip_radius_rel_err": abs(f32[-1, 3] - f64[-1, 3]) / f64[-1, 3],
        "solute_rel_diff": abs(f32[-1, 4] - f64[-1, 4]) / abs(f64[-1, 4]),
        "solid_fraction_fp64": f64[-1, 5], "nonfinite": int(f32[:, 6].max() + f64[:, 6].max()),
        "wall_s": time.time() - t0,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=50000)
    ap.add_argument("--every", type=int, default=1000)
    a = ap.parse_args()
    print(json.dumps(compare(a.mesh, a.steps, a.every)))


if __name__ == "__main__":
    main()
