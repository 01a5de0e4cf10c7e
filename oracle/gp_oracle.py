"""ctypes front end of the CPU oracle (gp_oracle.c) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module; it is the checker, never the thing measured or shipped.

The oracle works on the reference's ghost-padded layout: planes of
(MESH_X+6) x (MESH_Y+6) doubles, index y + x*(MESH_Y+6), phases first, then the
K-1 chemical potentials.  `OracleModel` carries the model constants in the
reference's own units (the names follow functions/global_vars.h of
Grand_potential_Finite_difference_2D_serial).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libgp_oracle.so")
HARNESS_PATH = os.path.join(HERE, "_ref", "gp_ref_harness")


class _Params(C.Structure):
    _fields_ = [
        ("N", C.c_int), ("K1", C.c_int),
        ("mesh_x", C.c_long), ("mesh_y", C.c_long),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double),
        ("epsilon", C.c_double), ("tau", C.c_double), ("T", C.c_double), ("Teq", C.c_double),
        ("obstacle", C.c_int), ("anisotropy", C.c_int),
        ("binary", C.c_int), ("ternary", C.c_int), ("dilute", C.c_int),
        ("bc_phi", C.c_int * 4), ("bc_mu", C.c_int * 4),
        ("Gamma", C.c_void_p), ("Gamma_abc", C.c_void_p), ("tau_ab", C.c_void_p), ("dab", C.c_void_p),
        ("R", C.c_void_p), ("Rinv", C.c_void_p), ("cmu", C.c_void_p), ("A", C.c_void_p),
        ("Beq", C.c_void_p), ("dBbdT", C.c_void_p), ("B", C.c_void_p), ("C", C.c_void_p),
        ("Diff", C.c_void_p),
    ]


class _Stats(C.Structure):
    _fields_ = [(n, C.c_double * 8) for n in
                ("phi_max", "phi_min", "rel_change_phi", "mu_max", "mu_min", "rel_change_mu")]


_lib = None


def build(force: bool = False) -> str:
    """Compile the restatement (needs only this directory and gcc)."""
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < max(os.path.getmtime(os.path.join(HERE, f))
                                             for f in ("gp_oracle.c", "gp_oracle.h")):
        subprocess.run(["make", "-C", HERE, "restatement"], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        _lib.gpo_step.argtypes = [C.POINTER(_Params), C.c_void_p, C.c_void_p, C.c_long, C.c_void_p,
                                  C.POINTER(_Stats)]
        _lib.gpo_step.restype = C.c_int
        _lib.gpo_apply_bc.argtypes = [C.POINTER(_Params), C.c_void_p, C.c_void_p]
        _lib.gpo_apply_bc.restype = None
        _lib.gpo_smooth.argtypes = [C.POINTER(_Params), C.c_void_p, C.c_void_p, C.c_long]
        _lib.gpo_smooth.restype = C.c_int
    return _lib


@dataclass
class OracleModel:
    """Model constants of one instance (reference units and meaning)."""
    N: int
    K1: int
    mesh_x: int
    mesh_y: int
    dx: float
    dy: float
    dt: float
    epsilon: float
    tau: float
    T: float
    Teq: float
    obstacle: int
    anisotropy: int
    binary: int
    ternary: int
    dilute: int
    bc_phi: tuple
    bc_mu: tuple
    Gamma: np.ndarray
    tau_ab: np.ndarray
    cmu: np.ndarray
    A: np.ndarray
    Beq: np.ndarray
    dBbdT: np.ndarray
    B: np.ndarray
    C: np.ndarray
    Diff: np.ndarray
    dab: np.ndarray | None = None
    R: np.ndarray | None = None
    Rinv: np.ndarray | None = None
    Gamma_abc: np.ndarray | None = None
    _keep: list = field(default_factory=list, repr=False)

    def _arr(self, a, shape):
        if a is None:
            a = np.zeros(shape)
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))
        self._keep.append(a)
        return a.ctypes.data

    def params(self) -> _Params:
        N, K1 = self.N, self.K1
        self._keep = []
        p = _Params()
        p.N, p.K1 = N, K1
        p.mesh_x, p.mesh_y = self.mesh_x, self.mesh_y
        p.dx, p.dy, p.dt = self.dx, self.dy, self.dt
        p.epsilon, p.tau, p.T, p.Teq = self.epsilon, self.tau, self.T, self.Teq
        p.obstacle, p.anisotropy = self.obstacle, self.anisotropy
        p.binary, p.ternary, p.dilute = self.binary, self.ternary, self.dilute
        p.bc_phi = (C.c_int * 4)(*self.bc_phi)
        p.bc_mu = (C.c_int * 4)(*self.bc_mu)
        p.Gamma = self._arr(self.Gamma, (N, N))
        p.Gamma_abc = self._arr(self.Gamma_abc, (N, N, N))
        p.tau_ab = self._arr(self.tau_ab, (N, N))
        p.dab = self._arr(self.dab, (N, N))
        p.R = self._arr(self.R, (N, N, 3, 3))
        p.Rinv = self._arr(self.Rinv, (N, N, 3, 3))
        p.cmu = self._arr(self.cmu, (N, K1, K1))
        p.A = self._arr(self.A, (N, K1, K1))
        p.Beq = self._arr(self.Beq, (N, K1))
        p.dBbdT = self._arr(self.dBbdT, (N, K1))
        p.B = self._arr(self.B, (N, K1))
        p.C = self._arr(self.C, (N,))
        p.Diff = self._arr(self.Diff, (N, K1, K1))
        return p


def step(model: OracleModel, phi: np.ndarray, mu: np.ndarray, nsteps: int, want_dphi: bool = False,
         want_stats: bool = False):
    """Advance ghost-padded (phi[N,rx,ry], mu[K1,rx,ry]) in place by nsteps steps.

    Returns (dphi_first or None, stats dict or None)."""
    L = lib()
    assert phi.dtype == np.float64 and phi.flags.c_contiguous
    assert mu.dtype == np.float64 and mu.flags.c_contiguous
    p = model.params()
    dphi = np.zeros_like(phi) if want_dphi else None
    st = _Stats() if want_stats else None
    rc = L.gpo_step(C.byref(p), phi.ctypes.data, mu.ctypes.data, nsteps,
                    dphi.ctypes.data if dphi is not None else None,
                    C.byref(st) if st is not None else None)
    if rc != 0:
        raise ValueError("oracle rejected the parameters (rc=%d)" % rc)
    stats = None
    if st is not None:
        stats = {n: np.array(getattr(st, n)[: (model.N if "phi" in n else model.K1)])
                 for n, _ in _Stats._fields_}
    return dphi, stats


def smooth(model: OracleModel, phi: np.ndarray, mu: np.ndarray, nsteps: int) -> None:
    """nsteps smoothing pre-steps (the reference runs NSMOOTH - 1 of them,
    microsim_gp.c:97-100) on ghost-padded fields, in place."""
    assert phi.dtype == np.float64 and phi.flags.c_contiguous
    assert mu.dtype == np.float64 and mu.flags.c_contiguous
    p = model.params()
    rc = lib().gpo_smooth(C.byref(p), phi.ctypes.data, mu.ctypes.data, nsteps)
    if rc != 0:
        raise ValueError("oracle rejected the parameters (rc=%d)" % rc)


def apply_bc(model: OracleModel, phi: np.ndarray, mu: np.ndarray) -> None:
    p = model.params()
    lib().gpo_apply_bc(C.byref(p), phi.ctypes.data, mu.ctypes.data)


# ---------------------------------------------------------------------------
# Reading the reference harness's dumps (consts.txt, state_<t>.bin)
# ---------------------------------------------------------------------------

def read_consts(path: str) -> dict:
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            name, n = parts[0], int(parts[1])
            vals = np.array([float(v) for v in parts[2:2 + n]])
            out[name] = vals
    return out


def read_state(path: str):
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(32), dtype=np.int64)
        rx, ry, N, NC = (int(v) for v in hdr)
        body = np.frombuffer(f.read(), dtype=np.float64)
    if body.size == N * rx * ry:  # Delta-phi dump
        return body.reshape(N, rx, ry).copy(), None
    phi = body[: N * rx * ry].reshape(N, rx, ry).copy()
    mu = body[N * rx * ry:].reshape(NC - 1, rx, ry).copy()
    return phi, mu


def model_from_consts(c: dict) -> OracleModel:
    N = int(c["NUMPHASES"][0])
    K1 = int(c["NUMCOMPONENTS"][0]) - 1
    aniso = int(c["ANISOTROPY"][0])
    return OracleModel(
        N=N, K1=K1, mesh_x=int(c["MESH_X"][0]), mesh_y=int(c["MESH_Y"][0]),
        dx=c["deltax"][0], dy=c["deltay"][0], dt=c["deltat"][0], epsilon=c["epsilon"][0],
        tau=c["tau"][0], T=c["T"][0], Teq=c["Teq"][0], obstacle=int(c["OBSTACLE"][0]),
        anisotropy=aniso, binary=int(c["BINARY"][0]), ternary=int(c["TERNARY"][0]),
        dilute=int(c["DILUTE"][0]),
        bc_phi=tuple(int(v) for v in c["bc_phi"]), bc_mu=tuple(int(v) for v in c["bc_mu"]),
        Gamma=c["Gamma"].reshape(N, N), tau_ab=c["tau_ab"].reshape(N, N),
        cmu=c["cmu"].reshape(N, K1, K1), A=c["A"].reshape(N, K1, K1), Beq=c["Beq"].reshape(N, K1),
        dBbdT=c["dBbdT"].reshape(N, K1), B=c["B"].reshape(N, K1), C=c["C"].reshape(N),
        Diff=c["Diffusivity"].reshape(N, K1, K1),
        dab=c["dab"].reshape(N, N) if aniso else None,
        R=c["Rotation_matrix"].reshape(N, N, 3, 3) if aniso else None,
        Rinv=c["Inv_Rotation_matrix"].reshape(N, N, 3, 3) if aniso else None,
        Gamma_abc=c["Gamma_abc"].reshape(N, N, N) if "Gamma_abc" in c else None,
    )


def run_reference_harness(workdir: str, input_in: str, filling_in: str, nsteps: int, dump_steps=(),
                          dumpdir: str | None = None, timeout: float | None = None) -> str:
    """Run oracle/_ref/gp_ref_harness (the reference compiled from source) in workdir.
    Returns its stdout."""
    args = [HARNESS_PATH, input_in, filling_in, "out", dumpdir or "-", str(nsteps)] + [str(s) for s in dump_steps]
    r = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference harness failed: %s" % r.stderr[-2000:])
    return r.stdout


# ---------------------------------------------------------------------------
# Energies of a state (numpy, FP64): the checker of gp_stats' energy sums
# ---------------------------------------------------------------------------

def _bc_index(M: int, kind: int) -> np.ndarray:
    """Source interior index of every coordinate -1 .. M (the boundary copy of
    solverloop/boundary_serial.h:176-203 as an index map: Neumann mirrors about the
    first/last interior cell, the periodic copy has period M-1,
    functions/utility_functions.h:471-653)."""
    v = np.arange(-1, M + 1)
    out = v.copy()
    if kind == 1:
        out[v < 0] = -v[v < 0]
        out[v >= M] = 2 * M - 2 - v[v >= M]
    else:
        out[v < 0] = M - 1 + v[v < 0]
        out[v >= M] = 1 + v[v >= M] - M
    return out


def energies(c: dict, phi: np.ndarray, mu: np.ndarray) -> dict:
    """Integrated energies of interior fields phi[N, mx, my], mu[K1, mx, my].

    c holds the model: N, K1, dx, dy, epsilon, obstacle, anisotropy, bc_phi (x, y
    types), Gamma[N,N], Gamma_abc[N,N,N], dab[N,N], R[N,N,2,2], cmu[N,K1,K1],
    A[N,K1,K1], Beff[N,K1] (Beq + dBbdT (T - Teq)), B[N,K1], C[N].  Per cell, with
    cell-centred gradients (gradphi_c of solverloop/calculate_gradients.h:92-131):
      gradient   eps sum_{a<b} Gamma_ab a_c(R_ab q_ab)^2 |q_ab|^2,
                 q_ab = phi_a grad phi_b - phi_b grad phi_a
                 (function_A_00.h:4-23 is its phi-derivative; a_c of anisotropy_01.h:30-48)
      potential  (1/eps) [16/pi^2 sum_{a<b} Gamma_ab |phi_a phi_b|      (functionW_01.h:6-39)
                          or 9 sum_{a<b} Gamma_ab phi_a^2 phi_b^2      (functionW_02.h:4-33)
                          + sum_{a<b<c} Gamma_abc |phi_a phi_b phi_c|]
      chemical   sum_a h_a f_a(c_a(mu))      (functionF_01.h:5-18 free_energy, :30-40 c_mu, functionH.h)
      grand      gradient + potential + sum_a h_a (f_a - mu . c_a)   (the psi of functionF_01.h:41-57)
    Each sum is multiplied by dx * dy."""
    N, K1 = c["N"], c["K1"]
    mx, my = phi.shape[1], phi.shape[2]
    ix, iy = _bc_index(mx, c["bc_phi"][0]), _bc_index(my, c["bc_phi"][1])
    P = phi[:, ix][:, :, iy]  # ghost ring of one cell
    gx = (P[:, 2:, 1:-1] - P[:, :-2, 1:-1]) * (0.5 / c["dx"])
    gy = (P[:, 1:-1, 2:] - P[:, 1:-1, :-2]) * (0.5 / c["dy"])
    eg = np.zeros((mx, my))
    w2 = np.zeros((mx, my))
    w3 = np.zeros((mx, my))
    for a in range(N):
        for b in range(a + 1, N):
            Qx = phi[a] * gx[b] - phi[b] * gx[a]
            Qy = phi[a] * gy[b] - phi[b] * gy[a]
            ac = np.ones((mx, my))
            if c["anisotropy"]:
                R = c["R"][a][b]
                q0, q1 = R[0][0] * Qx + R[0][1] * Qy, R[1][0] * Qx + R[1][1] * Qy
                q2 = q0 * q0 + q1 * q1
                big = q2 > 1.0e-15
                s4 = np.where(big, (q0 ** 4 + q1 ** 4) / np.where(big, q2 * q2, 1.0), 0.0)
                ac = np.where(big, 1.0 - c["dab"][a][b] * (3.0 - 4.0 * s4), 1.0)
            eg += c["Gamma"][a][b] * ac * ac * (Qx * Qx + Qy * Qy)
            if c["obstacle"]:
                w2 += c["Gamma"][a][b] * np.abs(phi[a] * phi[b])
            else:
                w2 += c["Gamma"][a][b] * phi[a] ** 2 * phi[b] ** 2
            for d in range(b + 1, N):
                w3 += c["Gamma_abc"][a][b][d] * np.abs(phi[a] * phi[b] * phi[d])
    pot = (w2 * (16.0 / (np.pi * np.pi) if c["obstacle"] else 9.0) + w3) / c["epsilon"]
    fch = np.zeros((mx, my))
    psi = np.zeros((mx, my))
    for a in range(N):
        s1 = np.zeros((mx, my))
        for b in range(N):
            for d in range(b + 1, N):
                if a not in (b, d):
                    s1 += phi[b] * phi[d]
        h = phi[a] ** 2 * (3.0 - 2.0 * phi[a]) + 2.0 * phi[a] * s1
        conc = [sum(c["cmu"][a][k][l] * (mu[l] - c["Beff"][a][l]) for l in range(K1)) for k in range(K1)]
        f = np.full((mx, my), float(c["C"][a]))
        mc = np.zeros((mx, my))
        for k in range(K1):
            for l in range(k, K1):
                f += c["A"][a][k][l] * conc[k] * conc[l]
            f += c["B"][a][k] * conc[k]
            mc += mu[k] * conc[k]
        fch += h * f
        psi += h * (f - mc)
    da = c["dx"] * c["dy"]
    grad = c["epsilon"] * eg
    return {"energy_gradient": grad.sum() * da, "energy_potential": pot.sum() * da,
            "energy_chemical": fch.sum() * da, "grand_potential": (grad + pot + psi).sum() * da}
