"""Gradients of a field-mismatch loss through many explicit steps: a thin
binding of the C ABI's hand-written adjoint (gp_adj_*, binary alloys) and a
torch.autograd.Function around it.

Parameters (the order of gp_adj_backward's gradient):
  0  mobility M = 1 / tau_ab[0][1]   (the fallback tau is scaled with it)
  1  anisotropy strength dab[0][1]
  2  interface energy Gamma[0][1]
  3  liquid diffusivity Diff[1][0][0]

    params = torch.tensor(adjoint.params_of(model), dtype=torch.float64, requires_grad=True)
    phi = adjoint.GPSteps.apply(params, model, phi0, mu0, nsteps)      # final phi, [2, mx, my]
    loss = ((phi - target) ** 2).sum()
    loss.backward()                                                     # params.grad
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import GP_FP32, GP_FP64, GpModel, _check, _ptr, lib

NPARAM = 4
NAMES = ("mobility", "delta", "gamma", "D_liquid")


def params_of(m: GpModel) -> np.ndarray:
    """The four parameters of a binary model."""
    return np.array([1.0 / m.arr("tau_ab")[0, 1], m.arr("dab")[0, 1], m.arr("Gamma")[0, 1],
                     m.arr("Diff")[1, 0, 0]], dtype=np.float64)


def with_params(m: GpModel, p) -> GpModel:
    """A copy of m with the four parameters set (pairs kept symmetric, tau
    scaled with tau_ab)."""
    p = [float(v) for v in p]
    out = m.copy()
    tau_ab = out.arr("tau_ab")
    ratio = m.tau / m.arr("tau_ab")[0, 1]
    tau_ab[0, 1] = tau_ab[1, 0] = 1.0 / p[0]
    out.tau = ratio / p[0]
    dab = out.arr("dab")
    dab[0, 1] = dab[1, 0] = p[1]
    gam = out.arr("Gamma")
    gam[0, 1] = gam[1, 0] = p[2]
    out.arr("Diff")[1, 0, 0] = p[3]
    return out


class Adjoint:
    """One instance: forward with checkpoints, then the adjoint sweep."""

    def __init__(self, model: GpModel, precision: int = GP_FP64):
        self.model = model
        self._h = C.c_void_p()
        _check("gp_adj_create", lib().gp_adj_create(C.byref(model), precision, C.byref(self._h)))
        self.shape = (int(model.mesh_x), int(model.mesh_y))

    def close(self):
        if self._h:
            lib().gp_adj_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, phi0: np.ndarray, mu0: np.ndarray, nsteps: int, every: int = 0):
        """Run nsteps steps (checkpoint every `every` steps, 0: sqrt(nsteps));
        returns the final (phi [2, mx, my], mu [1, mx, my])."""
        mx, my = self.shape
        p0 = np.ascontiguousarray(phi0, dtype=np.float64).reshape(2, mx, my)
        u0 = np.ascontiguousarray(mu0, dtype=np.float64).reshape(1, mx, my)
        p = np.empty((2, mx, my))
        u = np.empty((1, mx, my))
        _check("gp_adj_forward", lib().gp_adj_forward(self._h, _ptr(p0), _ptr(u0), int(nsteps), int(every),
                                                      _ptr(p), _ptr(u)))
        return p, u

    def backward(self, lam_phi: np.ndarray, lam_mu: np.ndarray | None = None, initial: bool = False):
        """Gradient of the loss with respect to the four parameters, given its
        adjoint with respect to the final state; with initial=True also the
        adjoints of the initial phi and mu."""
        mx, my = self.shape
        lp = np.ascontiguousarray(lam_phi, dtype=np.float64).reshape(2, mx, my)
        lu = None if lam_mu is None else np.ascontiguousarray(lam_mu, dtype=np.float64).reshape(1, mx, my)
        g = np.zeros(NPARAM)
        p0 = np.empty((2, mx, my)) if initial else None
        u0 = np.empty((1, mx, my)) if initial else None
        _check("gp_adj_backward", lib().gp_adj_backward(self._h, _ptr(lp), None if lu is None else _ptr(lu),
                                                        _ptr(g), None if p0 is None else _ptr(p0),
                                                        None if u0 is None else _ptr(u0)))
        return (g, p0, u0) if initial else g

    @property
    def stored_states(self) -> int:
        n = C.c_int64()
        _check("gp_adj_stored_states", lib().gp_adj_stored_states(self._h, C.byref(n)))
        return n.value


def _torch_function():
    import torch

    class GPSteps(torch.autograd.Function):
        """phi after nsteps explicit steps as a function of the four parameters
        (forward and backward on the GPU through gp_adj_*)."""

        @staticmethod
        def forward(ctx, params, model, phi0, mu0, nsteps, precision=GP_FP64, every=0):
            adj = Adjoint(with_params(model, params.detach().cpu().numpy()), precision)
            phi, _ = adj.forward(phi0, mu0, nsteps, every)
            ctx.adj = adj
            return torch.from_numpy(phi).to(params.dtype)

        @staticmethod
        def backward(ctx, gphi):
            g = ctx.adj.backward(gphi.detach().cpu().numpy().astype(np.float64))
            ctx.adj.close()
            return (torch.from_numpy(g).to(gphi.dtype), None, None, None, None, None, None)

    return GPSteps


def __getattr__(name):
    if name == "GPSteps":
        return _torch_function()
    raise AttributeError(name)
