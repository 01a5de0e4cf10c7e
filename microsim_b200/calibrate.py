"""Adjoint calibration workload: gradients of a field-mismatch loss with
respect to mobility, anisotropy strength, interface energy and liquid
diffusivity, through the hand-written adjoint (gp_adj_*).

    python -m microsim_b200.calibrate [--instances 32] [--mesh 512] [--steps 2000] [--fd 1]

Each instance (binary anisotropic growth from a centred seed) gets a target
field from the forward run with perturbed parameters (mobility x1.1,
delta + 0.005, D_liquid x0.9); the loss is L = sum (phi_N - target)^2.  Every
instance's gradient is computed with the FP32 adjoint and the FP64 reference
adjoint (sqrt(N) checkpointing); the first `--fd` instances are also checked
against central finite differences of the FP64 forward (h = 1e-4 relative).
Prints one JSON line: per-parameter worst relative differences, the time of a
forward + backward per instance and the states stored.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import GP_FP32, GP_FP64, adjoint, configs, load_case


def run(instances: int = 32, mesh: int = 512, steps: int = 2000, fd: int = 1) -> dict:
    cases = configs.c5(n=instances, steps=steps, mesh=mesh)
    out = {"instances": instances, "mesh": mesh, "steps": steps, "fd_instances": fd}
    worst32 = np.zeros(adjoint.NPARAM)
    worstfd = np.zeros(adjoint.NPARAM)
    t32 = t64 = 0.0
    grads = []
    for i, case in enumerate(cases):
        m, phi, mu = load_case(case)
        p = adjoint.params_of(m)
        tm = adjoint.with_params(m, p * np.array([1.1, 1.0, 1.0, 0.9]) + np.array([0.0, 0.005, 0.0, 0.0]))
        with adjoint.Adjoint(tm, GP_FP64) as a:
            target, _ = a.forward(phi, mu, steps)
        g = {}
        for prec in (GP_FP32, GP_FP64):
            t0 = time.time()
            with adjoint.Adjoint(m, prec) as a:
                ph, _ = a.forward(phi, mu, steps)
                g[prec] = a.backward(2.0 * (ph - target))
                out["stored_states"] = a.stored_states
            dt = time.time() - t0
            if prec == GP_FP32:
                t32 += dt
            else:
                t64 += dt
        worst32 = np.maximum(worst32, np.abs(g[GP_FP32] - g[GP_FP64]) / np.abs(g[GP_FP64]))
        grads.append(g[GP_FP64].tolist())
        if i < fd:
            def loss(params):
                with adjoint.Adjoint(adjoint.with_params(m, params), GP_FP64) as a:
                    q, _ = a.forward(phi, mu, steps)
                return float(((q - target) ** 2).sum())
            for k in range(adjoint.NPARAM):
                h = 1e-4 * abs(p[k])
                pp, pm = p.copy(), p.copy()
                pp[k] += h
                pm[k] -= h
                fdk = (loss(pp) - loss(pm)) / (2 * h)
                worstfd[k] = max(worstfd[k], abs(g[GP_FP64][k] - fdk) / abs(fdk))
                out.setdefault("fd_gradient", []).append(fdk)
    out.update({
        "fp32_vs_fp64_rel": dict(zip(adjoint.NAMES, worst32.tolist())),
        "fp64_vs_fd_rel": dict(zip(adjoint.NAMES, worstfd.tolist())) if fd else None,
        "gradient_first_instance": dict(zip(adjoint.NAMES, grads[0])),
        "seconds_per_instance_fp32": t32 / instances,
        "seconds_per_instance_fp64": t64 / instances,
    })
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=32)
    ap.add_argument("--mesh", type=int, default=512)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--fd", type=int, default=1)
    a = ap.parse_args()
    print(json.dumps(run(a.instances, a.mesh, a.steps, a.fd)))


if __name__ == "__main__":
    main()
