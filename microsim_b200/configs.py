"""Input.in / Filling.in writer and the named synthetic workloads.

The files follow the grammar of the reference's parser
(Grand_potential_Finite_difference_2D_serial/functions/reading_input_parameters.h):
one ``KEY = VALUE;`` per line, keys in an order the parser accepts
(DIMENSION and NUMPHASES/NUMCOMPONENTS before any matrix, Function_anisotropy
before Anisotropy_type/Rotation_matrix, Shift before Shiftj, BOUNDARY before
BOUNDARY_VALUE), no blank lines (the reference re-applies the previous key on a
blank line).  The reference copies each ``{a,b,c}`` token into a 10-byte buffer,
so every token written here is at most 9 characters and has no blank.

Workloads (interior sizes, the reference's units):

* ``c1``   200x200, 2 phases, binary, isotropic, obstacle, seed r=10 at the
  centre, dt = 0.2 dx^2/(4D) = 0.05, 10,000 steps (literal parameters: the
  reference itself is unstable at this dt and produces a checkerboard);
* ``c1g``  the same with a 10x larger composition gap (ceq +-0.5, cfill -0.2,
  tau 1.7776): a seed that grows, for tip and mass measurements;
* ``c2``   1024x1024 4-fold dendrite (delta = 0.02), seed r=8 at the corner
  with mirror boundaries, 50,000 steps (``c2g``: growing-gap variant);
* ``c3``   2048x2048, 4 phases (3 rotated solid grains + liquid), ternary,
  64 seeds, delta = 0.01, 20,000 steps;
* ``c4``   256 independent binary dendrites, sides in {128..512}, 5,000 steps;
* ``c5``   32 x 512^2 binary anisotropic instances, 2,000 steps.
Seeds come from numpy's default_rng with fixed seeds.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


def fmt(v) -> str:
    """Shortest number text of at most 9 characters that atof reads back."""
    if isinstance(v, (int, np.integer)):
        s = str(int(v))
    else:
        v = float(v)
        s = None
        for prec in range(9, 0, -1):
            t = ("%." + str(prec) + "g") % v
            if "e" in t:
                m, e = t.split("e")
                t = m + "e" + str(int(e))
            if len(t) <= 9:
                s = t
                break
    if s is None or len(s) > 9:
        raise ValueError(f"value {v!r} does not fit the reference's 9-character tokens")
    return s


def brace(vals) -> str:
    return "{" + ",".join(fmt(v) for v in vals) + "}"


@dataclass
class Case:
    """Everything an Input.in / Filling.in pair says, in the reference's terms."""
    mesh_x: int = 200
    mesh_y: int = 200
    dx: float = 1.0
    dt: float = 0.05
    N: int = 2
    K: int = 2                      # NUMCOMPONENTS
    ntimesteps: int = 1000
    savet: int = 1000
    nsmooth: int = 1
    shift: int = 0                  # moving frame along +y (Shift / Shiftj)
    shiftj: int = 0
    track: int = 1000
    epsilon: float = 4.0
    tau: float = 1.0                # FunctionTau fallback
    gamma: list = field(default_factory=lambda: [1.0])          # pairs (a<b)
    tau_ab: list = field(default_factory=lambda: [1.0])         # pairs (a<b)
    aniso: int = 0
    dab: list = field(default_factory=lambda: [0.0])            # pairs (a<b)
    rotations: list = field(default_factory=list)              # (a, b, theta_z deg)
    function_w: int = 1
    gamma_abc: list = field(default_factory=list)              # triples (a<b<c)
    diffusivity: list = field(default_factory=list)            # (diag flag, phase, values...)
    A: list = field(default_factory=list)                      # (phase, diag..., offdiag...)
    ceq: list = field(default_factory=list)                    # (p1, p2, values...)
    cfill: list = field(default_factory=list)
    slopes: list = field(default_factory=list)
    T: float = 1.0
    Teq: float = 1.0
    Tfill: float = 1.0
    bc_phi: tuple = (1, 1, 1, 1)    # X+, X-, Y+, Y- as written in Input.in
    bc_mu: tuple = (1, 1, 1, 1)
    solver: str | None = "BINARY"   # BINARY / TERNARY / DILUTE / None (LU)
    phases: list = field(default_factory=list)
    components: list = field(default_factory=list)
    writeformat: str = "BINARY"
    writecomposition: int = 0
    # frozen temperature gradient (ISOTHERMAL = 0): (base_temp, DeltaT, Distance, gradient_OFFSET,
    # velocity) and the temperature's boundary types (X+, X-, Y+, Y-); None: isothermal
    tempgrady: tuple | None = None
    bc_T: tuple | None = None
    fills: list = field(default_factory=list)                  # ("FILLCYLINDER", [..]) ...

    def input_text(self) -> str:
        N, K = self.N, self.K
        phases = self.phases or [f"p{i}" for i in range(N - 1)] + ["liquid"]
        comps = self.components or ["A", "B", "C", "D", "E"][:K]
        L = [
            "DIMENSION = 2;",
            f"MESH_X = {self.mesh_x};",
            f"MESH_Y = {self.mesh_y};",
            "MESH_Z = 1;",
            f"DELTA_X = {fmt(self.dx)};",
            f"DELTA_Y = {fmt(self.dx)};",
            f"DELTA_Z = {fmt(self.dx)};",
            f"DELTA_t = {fmt(self.dt)};",
            f"NUMPHASES = {N};",
            f"NUMCOMPONENTS = {K};",
            f"NTIMESTEPS = {self.ntimesteps};",
            f"NSMOOTH = {self.nsmooth};",
            f"SAVET = {self.savet};",
            "STARTTIME = 0;",
            "RESTART = 0;",
            "COMPONENTS = {" + ",".join(comps) + "};",
            "PHASES = {" + ",".join(phases) + "};",
            f"GAMMA = {brace(self.gamma)};",
        ]
        for d in self.diffusivity:
            L.append(f"DIFFUSIVITY = {brace(d)};")
        L += ["R = 1.0;", "V = 1.0;"]
        for name, t in (("phi", self.bc_phi), ("mu", self.bc_mu), ("c", self.bc_mu),
                        ("T", self.bc_T or self.bc_mu)):
            L.append("BOUNDARY = {" + name + "," + ",".join(str(v) for v in t) + ",0,0};")
        for name in ("phi", "mu", "c", "T"):
            L.append("BOUNDARY_VALUE = {" + name + ",0,0,0,0,0,0};")
        if self.tempgrady is None:
            L.append("ISOTHERMAL = 1;")
        else:
            L.append("ISOTHERMAL = 0;")
            L.append(f"Tempgrady = {brace(self.tempgrady)};")
        if self.solver:
            L.append(f"{self.solver} = 1;")
        L += [
            f"T = {fmt(self.T)};",
            f"WRITEFORMAT = {self.writeformat};",
            f"TRACK_PROGRESS = {self.track};",
            f"epsilon = {fmt(self.epsilon)};",
            f"tau = {fmt(self.tau)};",
            f"Tau = {brace(self.tau_ab)};",
            f"Function_anisotropy = {self.aniso};",
            "Anisotropy_type = 4;",
            f"dab = {brace(self.dab)};",
        ]
        for (a, b, th) in self.rotations:
            L.append(f"Rotation_matrix = {brace([a, b, 0, 0, th])};")
        L.append(f"Function_W = {self.function_w};")
        L.append("Gamma_abc = {" + ",".join(fmt(v) for v in self.gamma_abc) + "};")
        L += [
            f"Shift = {self.shift};",
            f"Shiftj = {self.shiftj};",
            f"Writecomposition = {self.writecomposition};",
            "Noise_phasefield = 0;",
            f"Equilibrium_temperature = {fmt(self.Teq)};",
            f"Filling_temperature = {fmt(self.Tfill)};",
            "Function_F = 1;",
        ]
        for a in self.A:
            L.append(f"A = {brace(a)};")
        for key, rows in (("ceq", self.ceq), ("cfill", self.cfill), ("slopes", self.slopes)):
            for r in rows:
                L.append(f"{key} = {brace(r)};")
        return "\n".join(L) + "\n"

    def filling_text(self) -> str:
        return "".join(f"{kind} = {brace(vals)};\n" for kind, vals in self.fills)

    def write(self, dirpath: str, stem: str = "Input"):
        os.makedirs(dirpath, exist_ok=True)
        ip = os.path.join(dirpath, f"{stem}.in")
        fp = os.path.join(dirpath, f"{stem.replace('Input', 'Filling')}.in" if stem != "Input" else "Filling.in")
        with open(ip, "w") as f:
            f.write(self.input_text())
        with open(fp, "w") as f:
            f.write(self.filling_text())
        return ip, fp

    @property
    def cells(self) -> int:
        return self.mesh_x * self.mesh_y


def binary_case(mesh_x, mesh_y, *, gap=0.1, supersat=0.3, eps=4.0, gamma=1.0, delta=0.0, theta=0.0,
                D_l=1.0, D_s=0.0, dt=None, tau=None, function_w=1, seed=(None, None, 10.0),
                bc=(1, 1, 1, 1), steps=1000, savet=None) -> Case:
    """Binary alloy, 2 phases, quadratic free energies with A_s = A_l = 1.

    The reference parametrises f_a(c) = A c^2 + B_a c + C_a with B = C = 0 for
    the liquid, so the configuration's f_s = c^2, f_l = c^2 + 2*gap*c is written
    as ceq_s = +gap/2, ceq_l = -gap/2 (mu shifted by a constant).  Supersaturation
    Omega puts the far-field liquid at cfill = ceq_l + Omega*gap.  tau defaults to the
    thin-interface relation tau = gap^2/(D_l/2) * eps * 0.2222 of the MPI twin's
    Calculate_Tau; dt defaults to 0.2 dx^2/(4 D_l)."""
    ceq_s, ceq_l = gap / 2.0, -gap / 2.0
    # Omega = (c_l,eq - c_inf)/(c_l,eq - c_s,eq)  =>  c_inf = c_l,eq + Omega*(c_s,eq - c_l,eq)
    cfill_l = round(ceq_l + supersat * (ceq_s - ceq_l), 6)
    if tau is None:
        tau = round(gap * gap / (D_l * 0.5) * eps * 0.2222, 6)
    if dt is None:
        dt = 0.2 * 1.0 / (4.0 * D_l)
    xc, yc, r = seed
    if xc is None:
        xc, yc = mesh_x // 2, mesh_y // 2
    c = Case(mesh_x=mesh_x, mesh_y=mesh_y, dx=1.0, dt=dt, N=2, K=2, ntimesteps=steps,
             savet=savet or steps, track=savet or steps, epsilon=eps, tau=tau, gamma=[gamma], tau_ab=[tau],
             aniso=1 if delta > 0 else 0, dab=[delta], rotations=[(0, 1, theta)] if delta > 0 else [],
             function_w=function_w,
             diffusivity=[(1, 0, D_s), (1, 1, D_l)],
             A=[(0, 1.0), (1, 1.0)],
             ceq=[(0, 0, ceq_s), (0, 1, ceq_l), (1, 1, ceq_l), (1, 0, ceq_l)],
             cfill=[(0, 0, ceq_s), (0, 1, ceq_l), (1, 1, cfill_l), (1, 0, ceq_l)],
             slopes=[(0, 0, 0.45), (0, 1, 0.45), (1, 0, 0.45), (1, 1, 0.45)],
             bc_phi=bc, bc_mu=bc, solver="BINARY", phases=["solid", "liquid"], components=["A", "B"],
             fills=[("FILLCYLINDER", [0, xc, yc, 0, 0, r])])
    return c


def c1(literal: bool = True, steps: int = 10000) -> Case:
    """200x200 isotropic binary, seed r=10 at the centre."""
    if literal:
        return binary_case(200, 200, gap=0.1, supersat=0.3, eps=4.0, dt=0.05, steps=steps, seed=(100, 100, 10.0))
    return binary_case(200, 200, gap=1.0, supersat=0.2, eps=4.0, dt=0.05, tau=1.7776, steps=steps,
                       seed=(100, 100, 10.0))


def c2(literal: bool = False, steps: int = 50000, mesh: int = 1024) -> Case:
    """Single 4-fold dendrite from the corner (mirror boundaries give the full crystal)."""
    if literal:
        return binary_case(mesh, mesh, gap=0.1, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, steps=steps,
                           seed=(0, 0, 8.0))
    return binary_case(mesh, mesh, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                       steps=steps, seed=(0, 0, 8.0))


def c3(steps: int = 20000, mesh: int = 2048, nseeds: int = 64, rng_seed: int = 3) -> Case:
    """4 phases (3 solid grains + liquid), 3 components (2 independent mu), ternary."""
    rng = np.random.default_rng(rng_seed)
    N, K = 4, 3
    A = []
    for a in range(N):
        # SPD Hessian muc = [[2A11, A12], [A12, 2A22]] with eigenvalues in [0.5, 2]
        ev = rng.uniform(0.5, 2.0, 2)
        th = rng.uniform(0, math.pi)
        Q = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]])
        H = Q @ np.diag(ev) @ Q.T
        A.append((a, round(H[0, 0] / 2, 4), round(H[1, 1] / 2, 4), round(H[0, 1], 4)))
    gap = 1.0
    ceq, cfill, slopes = [], [], []
    for a in range(N - 1):
        cs = [round(0.5 * gap * ((a + 1) % 2), 4), round(0.5 * gap * ((a + 1) // 2 % 2), 4)]
        cl = [-0.25, -0.25]
        ceq += [(a, a, *cs), (a, N - 1, *cl), (N - 1, a, *cl)]
        cfill += [(a, a, *cs), (a, N - 1, *cl), (N - 1, a, *cl)]
        slopes += [(a, a, 0.45, 0.45), (a, N - 1, 0.45, 0.45), (N - 1, a, 0.45, 0.45)]
    ceq.append((N - 1, N - 1, -0.25, -0.25))
    cfill.append((N - 1, N - 1, -0.3, -0.3))
    slopes.append((N - 1, N - 1, 0.45, 0.45))
    thetas = [round(float(v), 3) for v in rng.uniform(0.0, 90.0, N - 1)]
    rot = []
    for a in range(N):
        for b in range(a + 1, N):
            th = thetas[a] if b == N - 1 else round((thetas[a] + thetas[b]) / 2.0, 3)
            rot.append((a, b, th))
    pairs = N * (N - 1) // 2
    dab = []
    for a in range(N):
        for b in range(a + 1, N):
            dab.append(0.01 if b == N - 1 else 0.0)
    fills = []
    xs = rng.integers(0, mesh, nseeds)
    ys = rng.integers(0, mesh, nseeds)
    rs = rng.uniform(4.0, 12.0, nseeds)
    ph = rng.integers(0, N - 1, nseeds)
    ph[: N - 1] = np.arange(N - 1)  # every solid phase appears at least once
    for i in range(nseeds):
        fills.append(("FILLCYLINDER", [int(ph[i]), int(xs[i]), int(ys[i]), 0, 0, round(float(rs[i]), 3)]))
    D = [(1, a, 0.0, 0.0) for a in range(N - 1)] + [(1, N - 1, 1.0, 1.0)]
    return Case(mesh_x=mesh, mesh_y=mesh, dx=1.0, dt=0.04, N=N, K=K, ntimesteps=steps, savet=steps, track=steps,
                epsilon=4.0, tau=1.0, gamma=[1.0] * pairs, tau_ab=[1.0] * pairs, aniso=1, dab=dab, rotations=rot,
                function_w=1, gamma_abc=[5.0] * (N * (N - 1) * (N - 2) // 6), diffusivity=D, A=A, ceq=ceq,
                cfill=cfill, slopes=slopes, solver="TERNARY", phases=["g1", "g2", "g3", "liquid"],
                components=["Al", "Cu", "Ni"], fills=fills)


C4_SIDES = (128, 192, 256, 384, 512)


def c4(n: int = 256, steps: int = 5000, rng_seed: int = 4):
    """256 independent binary dendrites of uneven sizes and parameters."""
    rng = np.random.default_rng(rng_seed)
    out = []
    for i in range(n):
        side = int(rng.choice(C4_SIDES))
        delta = round(float(rng.uniform(0.0, 0.05)), 4)
        om = round(float(rng.uniform(0.3, 0.6)), 4)
        eps = float(rng.choice([3.0, 4.0, 5.0]))
        tau = round(1.0 * 1.0 / 0.5 * eps * 0.2222, 4)
        out.append(binary_case(side, side, gap=1.0, supersat=om, eps=eps, delta=delta, dt=0.05, tau=tau,
                               steps=steps, seed=(0, 0, 8.0)))
    return out


def c5(n: int = 32, steps: int = 2000, mesh: int = 512):
    """Adjoint calibration instances: binary anisotropic growth on 512^2."""
    return [binary_case(mesh, mesh, gap=1.0, supersat=0.5, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                        steps=steps, seed=(mesh // 2, mesh // 2, 10.0)) for _ in range(n)]
