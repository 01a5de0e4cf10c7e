"""A few FP32 batch steps of a bench workload inside an NVTX range named
"profile", for profilers (ncu --nvtx --nvtx-include "profile/").

    python -m microsim_b200.profile_step [--workload c4|c2|c1] [--state FILE]
                                         [--tile TX TY] [--steps S] [--full]
                                         [--depth 1|2] [--lean-per-sm L] [--general-per-sm G]
                                         [--compensated 0|1] [--fp64]

The workload's state is first advanced as the benchmark does (the batched
sweep 2,500 steps, the 1024^2 dendrite 25,000, the 200^2 seed 5,000); with
--state the advanced state is saved to FILE on the first run and read back on
later ones, so a profiled run launches only a handful of kernels before the
range.  --full switches the narrow band off (every tile through the full
kernel); --depth 2 steps in blocked pairs (two steps per lean box);
--lean-per-sm and --general-per-sm set the lean and full kernels' blocks per
SM (0: occupancy); --compensated 1 the compensated FP32 accumulation (default
0, plain, as the benchmark's headline); --fp64
profiles the plain FP64 step of the workload's first instance instead.
"""
from __future__ import annotations

import argparse
import os

import numpy as np


def main(argv=None):
    import torch
    import microsim_b200 as mb
    from microsim_b200 import configs

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c4", choices=["c1", "c2", "c4"])
    ap.add_argument("--state", default=None)
    ap.add_argument("--tile", type=int, nargs=2, default=[16, 32])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--full", action="store_true")
    ap.add_argument("--depth", type=int, default=1, choices=[1, 2])
    ap.add_argument("--lean-per-sm", type=int, default=0)
    ap.add_argument("--general-per-sm", type=int, default=0)
    ap.add_argument("--compensated", type=int, default=0, choices=[0, 1])
    ap.add_argument("--fp64", action="store_true")
    a = ap.parse_args(argv)
    cases = {"c4": configs.c4, "c2": lambda: [configs.c2(literal=False, steps=50000)],
             "c1": lambda: [configs.c1(literal=False, steps=10000)]}[a.workload]()
    loaded = [mb.load_case(c) for c in cases]
    models = [m for m, _, _ in loaded]
    if a.state and os.path.exists(a.state):
        z = np.load(a.state)
        fields = [(z[f"p{i}"], z[f"u{i}"]) for i in range(len(models))]
    else:
        prep = {"c4": 2500, "c2": 25000, "c1": 5000}[a.workload]
        with mb.Batch(models) as b:
            b.set_compensated(a.compensated == 1)
            for i, (_, p, u) in enumerate(loaded):
                b.upload(i, p, u)
            b.step(prep)
            fields = [b.download(i) for i in range(len(models))]
        if a.state:
            np.savez(a.state, **{f"p{i}": f[0] for i, f in enumerate(fields)},
                     **{f"u{i}": f[1] for i, f in enumerate(fields)})
    if a.fp64:
        with mb.Context(models[0], mb.GP_FP64) as c:
            c.upload(*fields[0])
            c.step(3)
            c.sync()
            torch.cuda.nvtx.range_push("profile")
            c.step(a.steps)
            c.sync()
            torch.cuda.nvtx.range_pop()
        print(f"profiled {a.steps} FP64 steps of {a.workload} instance 0 "
              f"({models[0].mesh_x}x{models[0].mesh_y})")
        return
    with mb.Batch(models) as b:
        b.set_tile(*a.tile)
        b.set_narrowband(not a.full)
        if not a.full:
            b.set_depth(a.depth)
        b.set_grids(a.lean_per_sm, a.general_per_sm)
        b.set_compensated(a.compensated == 1)
        for i, f in enumerate(fields):
            b.upload(i, *f)
        b.step(3)
        b.sync()
        torch.cuda.nvtx.range_push("profile")
        b.step(a.steps)
        b.sync()
        torch.cuda.nvtx.range_pop()
        lean, total, _ = b.lean_stats()
    print(f"profiled {a.steps} steps of {a.workload}, tile {a.tile[0]}x{a.tile[1]}, depth {a.depth}, "
          f"lean tiles {lean} of {total}")


if __name__ == "__main__":
    main()
