"""Generate the golden fixtures of tests/golden/ by running the reference itself.

Run here (where the reference tree is mounted), not on the GPU box:

    make -C oracle reference           # builds oracle/_ref/gp_ref_harness from the reference sources
    python tests/golden/make_golden.py

For every case below it writes Input.in / Filling.in with microsim_b200.configs,
runs the reference serial solver (compiled unchanged, driven by
oracle/ref_harness.c) and stores in tests/golden/<case>.npz:
  input_text, filling_text       the input files
  c_<name>                       the reference's model constants after init
  phi_<t>, mu_<t>                ghost-padded fields after step t (t = 0 and the dump steps)
  dphi_1                         Delta-phi after the phase-field half step of step 1
  vtk_0                          bytes of DATA/out_0.vtk from the reference's own writer
  stats                          the reference's running max/min/rel-change at the end
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from microsim_b200 import configs  # noqa: E402
from oracle import gp_oracle as O  # noqa: E402


def cases():
    C = configs
    out = {}
    # isotropic, obstacle, binary, Neumann, growing seed
    c = C.binary_case(24, 20, gap=1.0, supersat=0.3, eps=4.0, dt=0.05, tau=1.7776, seed=(12, 10, 5.0), steps=60)
    out["iso_obst_bin"] = (c, [1, 30, 60])
    # anisotropic (4-fold), obstacle, periodic x / Neumann y, corner seed
    c = C.binary_case(32, 24, gap=1.0, supersat=0.5, eps=4.0, delta=0.04, dt=0.05, tau=1.7776,
                      seed=(0, 0, 6.0), steps=60, bc=(3, 3, 1, 1))
    out["aniso_obst_bin_per"] = (c, [1, 30, 60])
    # anisotropic with a rotated frame, well potential, ASCII output with composition
    c = C.binary_case(24, 24, gap=1.0, supersat=0.4, eps=4.0, delta=0.03, theta=25.0, dt=0.05, tau=1.7776,
                      function_w=2, seed=(12, 12, 6.0), steps=60)
    c.writeformat = "ASCII"
    c.writecomposition = 1
    out["aniso_rot_well"] = (c, [1, 30, 60])
    # literal config-1 parameters on a small grid: explicitly unstable, all cells active
    c = C.binary_case(40, 40, gap=0.1, supersat=0.3, eps=4.0, dt=0.05, seed=(20, 20, 10.0), steps=30)
    out["c1_literal_small"] = (c, [1, 15, 30])
    # three phases, binary alloy, anisotropic with rotations on all pairs, third-order potential
    c = configs.Case(mesh_x=28, mesh_y=24, dx=1.0, dt=0.04, N=3, K=2, ntimesteps=40, epsilon=4.0, tau=1.0,
                     gamma=[1.0, 1.0, 1.0], tau_ab=[1.5, 1.5, 1.5], aniso=1, dab=[0.0, 0.03, 0.03],
                     rotations=[(0, 1, 0.0), (0, 2, 10.0), (1, 2, 40.0)], function_w=1, gamma_abc=[5.0],
                     diffusivity=[(1, 0, 0.0), (1, 1, 0.0), (1, 2, 1.0)], A=[(0, 1.0), (1, 1.0), (2, 1.0)],
                     ceq=[(0, 0, 0.78), (0, 2, 0.5), (2, 0, 0.5), (1, 1, 0.21), (1, 2, 0.5), (2, 1, 0.5),
                          (2, 2, 0.5)],
                     cfill=[(0, 0, 0.78), (0, 2, 0.5), (2, 0, 0.5), (1, 1, 0.21), (1, 2, 0.5), (2, 1, 0.5),
                            (2, 2, 0.45)],
                     slopes=[(0, 0, 0.45), (0, 2, 0.45), (2, 0, 0.45), (1, 1, -0.45), (1, 2, -0.45),
                             (2, 1, -0.45)],
                     T=0.98, bc_phi=(3, 3, 1, 1), bc_mu=(3, 3, 1, 1), solver="BINARY",
                     phases=["alpha", "beta", "liquid"], components=["Al", "Cu"],
                     fills=[("FILLCUBE", [0, 0, 0, 0, 13, 5, 0]), ("FILLCUBE", [1, 14, 0, 0, 27, 5, 0])])
    out["three_phase_eutectic"] = (c, [1, 20, 40])
    # four phases, ternary closed form, non-diagonal A, rotated grains
    c = C.c3(steps=40, mesh=32, nseeds=5, rng_seed=11)
    c.mesh_y = 28
    out["four_phase_ternary"] = (c, [1, 20, 40])
    # three components without a solver flag: the reference's LU inverse, isotropic, well
    c = configs.Case(mesh_x=20, mesh_y=20, dx=1.0, dt=0.04, N=2, K=3, ntimesteps=40, epsilon=4.0, tau=1.0,
                     gamma=[1.0], tau_ab=[1.2], aniso=0, dab=[0.0], function_w=2,
                     diffusivity=[(1, 0, 0.1, 0.1), (1, 1, 1.0, 0.8)],
                     A=[(0, 1.0, 1.2, 0.3), (1, 0.9, 1.0, -0.2)],
                     ceq=[(0, 0, 0.3, 0.2), (0, 1, -0.2, -0.1), (1, 1, -0.2, -0.1), (1, 0, -0.2, -0.1)],
                     cfill=[(0, 0, 0.3, 0.2), (0, 1, -0.2, -0.1), (1, 1, -0.1, -0.05), (1, 0, -0.2, -0.1)],
                     slopes=[(0, 0, 0.45, 0.3), (0, 1, 0.45, 0.3), (1, 0, 0.45, 0.3), (1, 1, 0.45, 0.3)],
                     solver=None, phases=["sol", "liq"], components=["X", "Y", "Z"],
                     fills=[("FILLCYLINDER", [0, 10, 10, 0, 0, 5.5])])
    out["lu_three_comp"] = (c, [1, 20, 40])
    # dilute solver, three phases, three components, isotropic obstacle
    c = configs.Case(mesh_x=24, mesh_y=20, dx=1.0, dt=0.04, N=3, K=3, ntimesteps=40, epsilon=4.0, tau=1.0,
                     gamma=[1.0, 1.2, 0.8], tau_ab=[1.0, 1.1, 1.3], aniso=0, dab=[0.0, 0.0, 0.0],
                     function_w=1, gamma_abc=[3.0],
                     diffusivity=[(1, 0, 0.0, 0.0), (1, 1, 0.0, 0.0), (1, 2, 1.0, 0.7)],
                     A=[(0, 1.0, 1.0, 0.0), (1, 1.0, 1.0, 0.0), (2, 1.0, 1.0, 0.0)],
                     ceq=[(0, 0, 0.4, 0.1), (0, 2, -0.2, -0.2), (2, 0, -0.2, -0.2), (1, 1, 0.1, 0.4),
                          (1, 2, -0.2, -0.2), (2, 1, -0.2, -0.2), (2, 2, -0.2, -0.2)],
                     cfill=[(0, 0, 0.4, 0.1), (0, 2, -0.2, -0.2), (2, 0, -0.2, -0.2), (1, 1, 0.1, 0.4),
                            (1, 2, -0.2, -0.2), (2, 1, -0.2, -0.2), (2, 2, -0.1, -0.1)],
                     slopes=[(0, 0, 0.45, 0.45), (0, 2, 0.45, 0.45), (2, 0, 0.45, 0.45), (1, 1, 0.45, 0.45),
                             (1, 2, 0.45, 0.45), (2, 1, 0.45, 0.45)],
                     solver="DILUTE", phases=["a", "b", "l"], components=["X", "Y", "Z"],
                     fills=[("FILLCYLINDER", [0, 7, 10, 0, 0, 4.0]), ("FILLSPHERE", [1, 17, 10, 0, 4.5])])
    out["dilute_three_phase"] = (c, [1, 20, 40])
    # smoothing pre-steps (NSMOOTH - 1 of them before the time loop): anisotropic obstacle binary
    c = C.binary_case(32, 28, gap=1.0, supersat=0.5, eps=4.0, delta=0.04, theta=15.0, dt=0.05, tau=1.7776,
                      seed=(16, 14, 6.0), steps=30)
    c.nsmooth = 8
    out["smooth_aniso_obst"] = (c, [1, 15, 30])
    # smoothing with three phases, well potential, periodic x
    c = configs.Case(mesh_x=28, mesh_y=24, dx=1.0, dt=0.04, N=3, K=2, ntimesteps=30, epsilon=4.0, tau=1.0,
                     gamma=[1.0, 1.0, 1.0], tau_ab=[1.5, 1.5, 1.5], aniso=0, dab=[0.0, 0.0, 0.0],
                     function_w=2, gamma_abc=[5.0],
                     diffusivity=[(1, 0, 0.0), (1, 1, 0.0), (1, 2, 1.0)], A=[(0, 1.0), (1, 1.0), (2, 1.0)],
                     ceq=[(0, 0, 0.78), (0, 2, 0.5), (2, 0, 0.5), (1, 1, 0.21), (1, 2, 0.5), (2, 1, 0.5),
                          (2, 2, 0.5)],
                     cfill=[(0, 0, 0.78), (0, 2, 0.5), (2, 0, 0.5), (1, 1, 0.21), (1, 2, 0.5), (2, 1, 0.5),
                            (2, 2, 0.45)],
                     slopes=[(0, 0, 0.45), (0, 2, 0.45), (2, 0, 0.45), (1, 1, -0.45), (1, 2, -0.45),
                             (2, 1, -0.45)],
                     T=0.98, bc_phi=(3, 3, 1, 1), bc_mu=(3, 3, 1, 1), solver="BINARY",
                     phases=["alpha", "beta", "liquid"], components=["Al", "Cu"],
                     fills=[("FILLCUBE", [0, 0, 0, 0, 13, 5, 0]), ("FILLCUBE", [1, 14, 0, 0, 27, 5, 0])])
    c.nsmooth = 6
    out["smooth_three_phase_well"] = (c, [1, 15, 30])
    # moving frame: a planar solid front growing along +y, the window shifted every 100 steps
    c = C.binary_case(24, 48, gap=1.0, supersat=0.6, eps=4.0, delta=0.02, dt=0.05, tau=1.7776, steps=400)
    c.fills = [("FILLCUBE", [0, 0, 0, 0, 23, 14, 0])]
    c.shift, c.shiftj = 1, 20
    out["shift_planar"] = (c, [1, 100, 200, 300, 400])
    # frozen temperature gradient (ISOTHERMAL = 0, Tempgrady): anisotropic obstacle binary, the
    # gradient moving along +y; ASCII output with composition and the Temperature field
    c = C.binary_case(32, 40, gap=1.0, supersat=0.5, eps=4.0, delta=0.03, theta=10.0, dt=0.05, tau=1.7776,
                      seed=(16, 10, 6.0), steps=60)
    c.tempgrady = (0.97, 0.08, 40.0, 2.0, 0.5)
    c.writeformat = "ASCII"
    c.writecomposition = 1
    out["tempgrad_aniso_bin"] = (c, [1, 30, 60])
    # frozen gradient, three phases, well potential, periodic x; the temperature's y ghosts not copied
    c = configs.Case(mesh_x=28, mesh_y=24, dx=1.0, dt=0.04, N=3, K=2, ntimesteps=40, epsilon=4.0, tau=1.0,
                     gamma=[1.0, 1.0, 1.0], tau_ab=[1.5, 1.5, 1.5], aniso=0, dab=[0.0, 0.0, 0.0],
                     function_w=2, gamma_abc=[5.0],
                     diffusivity=[(1, 0, 0.0), (1, 1, 0.0), (1, 2, 1.0)], A=[(0, 1.0), (1, 1.0), (2, 1.0)],
                     ceq=[(0, 0, 0.78), (0, 2, 0.5), (2, 0, 0.5), (1, 1, 0.21), (1, 2, 0.5), (2, 1, 0.5),
                          (2, 2, 0.5)],
                     cfill=[(0, 0, 0.78), (0, 2, 0.5), (2, 0, 0.5), (1, 1, 0.21), (1, 2, 0.5), (2, 1, 0.5),
                            (2, 2, 0.45)],
                     slopes=[(0, 0, 0.45), (0, 2, 0.45), (2, 0, 0.45), (1, 1, -0.45), (1, 2, -0.45),
                             (2, 1, -0.45)],
                     T=0.98, bc_phi=(3, 3, 1, 1), bc_mu=(3, 3, 1, 1), solver="BINARY",
                     phases=["alpha", "beta", "liquid"], components=["Al", "Cu"],
                     fills=[("FILLCUBE", [0, 0, 0, 0, 13, 5, 0]), ("FILLCUBE", [1, 14, 0, 0, 27, 5, 0])])
    c.tempgrady = (0.96, 0.05, 24.0, 0.0, 0.2)
    c.bc_T = (3, 3, 0, 0)
    out["tempgrad_three_phase_well"] = (c, [1, 20, 40])
    # the largest sizes the kernels take: six phases (five solid grains and the liquid), four
    # components (three independent mu, the reference's LU inverse), non-diagonal A, well potential
    # with the three-phase term, mixed boundaries
    N, K1 = 6, 3
    sol = list(range(N - 1))
    ceq, cfill, slopes = [], [], []
    for a in sol:
        cs = [round(0.1 + 0.05 * a, 2), round(0.3 - 0.04 * a, 2), round(0.05 + 0.03 * a, 2)]
        cl = [0.2, 0.15, 0.1]
        ceq += [(a, a, *cs), (a, N - 1, *cl), (N - 1, a, *cl)]
        cfill += [(a, a, *cs), (a, N - 1, *cl), (N - 1, a, *cl)]
        slopes += [(a, a, 0.45, 0.4, 0.35), (a, N - 1, 0.45, 0.4, 0.35), (N - 1, a, 0.45, 0.4, 0.35)]
    ceq.append((N - 1, N - 1, 0.2, 0.15, 0.1))
    cfill.append((N - 1, N - 1, 0.17, 0.12, 0.08))
    slopes.append((N - 1, N - 1, 0.45, 0.4, 0.35))
    pairs = N * (N - 1) // 2
    c = configs.Case(mesh_x=30, mesh_y=26, dx=1.0, dt=0.02, N=N, K=K1 + 1, ntimesteps=40, epsilon=4.0, tau=1.0,
                     gamma=[1.0 + 0.05 * i for i in range(pairs)], tau_ab=[1.2] * pairs, aniso=0, dab=[0.0] * pairs,
                     function_w=2, gamma_abc=[4.0] * (N * (N - 1) * (N - 2) // 6),
                     diffusivity=[(1, a, 0.05, 0.04, 0.03) for a in sol] + [(1, N - 1, 1.0, 0.8, 0.6)],
                     A=[(a, 1.0 + 0.1 * a, 1.1, 0.9, 0.1, -0.05, 0.08) for a in range(N)],
                     ceq=ceq, cfill=cfill, slopes=slopes, solver=None,
                     bc_phi=(3, 3, 1, 1), bc_mu=(3, 3, 1, 1),
                     phases=["g1", "g2", "g3", "g4", "g5", "liq"], components=["A", "B", "C", "D"],
                     fills=[("FILLCYLINDER", [0, 6, 6, 0, 0, 4.0]), ("FILLCYLINDER", [1, 22, 6, 0, 0, 4.5]),
                            ("FILLCYLINDER", [2, 15, 13, 0, 0, 5.0]), ("FILLCYLINDER", [3, 6, 20, 0, 0, 4.0]),
                            ("FILLCYLINDER", [4, 23, 20, 0, 0, 4.5])])
    out["six_phase_four_comp"] = (c, [1, 20, 40])
    return out


def run_case(name, case, dump_steps):
    with tempfile.TemporaryDirectory() as td:
        ip, fp = case.write(td)
        dd = os.path.join(td, "dump")
        os.makedirs(dd)
        nsteps = max(dump_steps)
        stdout = O.run_reference_harness(td, "Input.in", "Filling.in", nsteps, dump_steps, dumpdir=dd)
        data = {"input_text": np.array(case.input_text()), "filling_text": np.array(case.filling_text()),
                "dump_steps": np.array(dump_steps), "nonisothermal": np.array(int(case.tempgrady is not None))}
        for k, v in O.read_consts(os.path.join(dd, "consts.txt")).items():
            data["c_" + k] = v
        phi, mu = O.read_state(os.path.join(dd, "state_0.bin"))
        data["phi_0"], data["mu_0"] = phi, mu
        d, _ = O.read_state(os.path.join(dd, "dphi_1.bin"))
        data["dphi_1"] = d
        if case.nsmooth > 1:  # the state after the NSMOOTH - 1 smoothing pre-steps
            phi, mu = O.read_state(os.path.join(dd, "smoothed_0.bin"))
            data["phi_smoothed"], data["mu_smoothed"] = phi, mu
            data["nsmooth"] = np.array(case.nsmooth)
        for t in dump_steps:
            phi, mu = O.read_state(os.path.join(dd, f"state_{t}.bin"))
            data[f"phi_{t}"], data[f"mu_{t}"] = phi, mu
        with open(os.path.join(td, "DATA", "out_0.vtk"), "rb") as f:
            data["vtk_0"] = np.frombuffer(f.read(), dtype=np.uint8)
        shifts = [[int(v) for v in line.split()[1:]] for line in stdout.splitlines() if line.startswith("shift ")]
        if shifts:  # (step, interface row, accumulated offset) at every shift check
            data["shifts"] = np.array(shifts)
        stats = [line.split()[1:] for line in stdout.splitlines() if line.startswith("stat ")]
        data["stats"] = np.array([[float(v) for v in s[1:]] for s in stats])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
    return data


def main(only=None):
    if not os.path.exists(O.HARNESS_PATH):
        raise SystemExit("build the reference first: make -C oracle reference")
    for name, (case, steps) in cases().items():
        if only and name not in only:
            continue
        d = run_case(name, case, steps)
        size = os.path.getsize(os.path.join(HERE, name + ".npz"))
        print(f"{name}: N={case.N} K={case.K} {case.mesh_x}x{case.mesh_y} steps={steps} -> {size/1024:.1f} KiB")


if __name__ == "__main__" and len(sys.argv) == 1:
    main()
if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "only":
    main(sys.argv[2:])


# ---------------------------------------------------------------------------
# Long runs of the config-1 workload (200x200, 10,000 steps).  The final state is
# too large to commit; the fixture keeps one SHA-256 per x-row of the interior
# (phi planes then mu planes, little-endian float64 bytes) plus plane sums, so a
# bit-exact run can be checked and a mismatch localised to rows.
# ---------------------------------------------------------------------------

def row_digests(phi, mu):
    import hashlib
    planes = np.concatenate([phi, mu], axis=0)  # [N+K1, mx, my], interior
    return np.array([hashlib.sha256(np.ascontiguousarray(planes[:, x, :]).astype("<f8").tobytes()).hexdigest()
                     for x in range(planes.shape[1])])


def long_case(name, case, steps):
    with tempfile.TemporaryDirectory() as td:
        case.write(td)
        dd = os.path.join(td, "dump")
        os.makedirs(dd)
        O.run_reference_harness(td, "Input.in", "Filling.in", steps, [steps], dumpdir=dd)
        phi, mu = O.read_state(os.path.join(dd, f"state_{steps}.bin"))
    phi, mu = phi[:, 3:-3, 3:-3], mu[:, 3:-3, 3:-3]
    data = {"input_text": np.array(case.input_text()), "filling_text": np.array(case.filling_text()),
            "steps": np.array(steps), "row_sha256": row_digests(phi, mu),
            "plane_sums": np.concatenate([phi, mu]).sum(axis=(1, 2)),
            "plane_max": np.concatenate([phi, mu]).max(axis=(1, 2)),
            "plane_min": np.concatenate([phi, mu]).min(axis=(1, 2))}
    np.savez_compressed(os.path.join(HERE, name + ".long.npz"), **data)


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "long":
    which = sys.argv[2]
    if which == "c1_literal":
        long_case("c1_literal_10000", configs.c1(literal=True, steps=10000), 10000)
    elif which == "c1_growing":
        long_case("c1_growing_10000", configs.c1(literal=False, steps=10000), 10000)
