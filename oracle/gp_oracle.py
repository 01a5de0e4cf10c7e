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
