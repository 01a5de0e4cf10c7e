"""B200-native grand-potential explicit step (MicroSim GP solver drop-in).

Thin Python binding over the C ABI of ``include/gp_b200.h`` (``libgp_b200.so``,
built in-tree).  Everything that computes runs in that library: the host I/O
(Input.in / Filling.in / VTK with the reference's semantics) and the sm_100a
kernels.  There is no Python or CPU fallback: if the library is missing the
import of :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgp_b200.so")
DRIVER_PATH = os.path.join(HERE, "microsim_gp_b200")

GP_MAX_PHASES = 6
GP_MAX_K1 = 3
GP_NAME_LEN = 52

GP_OK, GP_E_ARG, GP_E_IO, GP_E_PARSE, GP_E_UNSUPPORTED, GP_E_CUDA, GP_E_NONFINITE, GP_E_NOMEM, \
    GP_E_TIMEOUT, GP_E_SIZE = 0, -1, -2, -3, -4, -5, -6, -7, -8, -9
GP_MU_BINARY, GP_MU_TERNARY, GP_MU_DILUTE, GP_MU_LU = 0, 1, 2, 3
GP_FP64, GP_FP32 = 0, 1
GP_BC_NEUMANN, GP_BC_PERIODIC = 1, 3
GP_STAT_VALUES = 64  # reduced FP64 values of one statistics read-back (include/gp_b200.h)

_P, _K = GP_MAX_PHASES, GP_MAX_K1


class GpModel(C.Structure):
    """ctypes mirror of ``gp_model`` (layout checked against gp_model_sizeof())."""
    _fields_ = [
        ("N", C.c_int32), ("K1", C.c_int32),
        ("mesh_x", C.c_int64), ("mesh_y", C.c_int64),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double),
        ("epsilon", C.c_double), ("tau", C.c_double), ("T", C.c_double), ("Teq", C.c_double),
        ("obstacle", C.c_int32), ("anisotropy", C.c_int32), ("mu_solver", C.c_int32),
        ("bc_phi", C.c_int32 * 4), ("bc_mu", C.c_int32 * 4), ("pad0", C.c_int32),
        ("Gamma", C.c_double * (_P * _P)),
        ("Gamma_abc", C.c_double * (_P * _P * _P)),
        ("tau_ab", C.c_double * (_P * _P)),
        ("dab", C.c_double * (_P * _P)),
        ("R", C.c_double * (_P * _P * 4)),
        ("Rinv", C.c_double * (_P * _P * 4)),
        ("cmu", C.c_double * (_P * _K * _K)),
        ("A", C.c_double * (_P * _K * _K)),
        ("Beff", C.c_double * (_P * _K)),
        ("Bfill", C.c_double * (_P * _K)),
        ("B", C.c_double * (_P * _K)),
        ("C", C.c_double * _P),
        ("Diff", C.c_double * (_P * _K * _K)),
        ("inv_eps", C.c_double), ("w_obstacle", C.c_double), ("jat_obst", C.c_double),
        ("jat_well", C.c_double), ("s_well", C.c_double),
        ("mu_shift", C.c_double * _K),
        ("nonisothermal", C.c_int32), ("bc_T", C.c_int32 * 4), ("pad1", C.c_int32),
        ("tg_base", C.c_double), ("tg_deltaT", C.c_double), ("tg_distance", C.c_double),
        ("tg_offset", C.c_double), ("tg_velocity", C.c_double),
        ("Beq", C.c_double * (_P * _K)), ("dBbdT", C.c_double * (_P * _K)),
        ("ceq_s", C.c_double * (_P * _K)), ("ceq_l", C.c_double * (_P * _K)), ("dC", C.c_double * (_P * _K)),
        ("dT_s", C.c_double * _P), ("dT_l", C.c_double * _P),
    ]

    def arr(self, name):
        """numpy view of an array field with its natural shape."""
        shapes = {"Gamma": (_P, _P), "Gamma_abc": (_P, _P, _P), "tau_ab": (_P, _P), "dab": (_P, _P),
                  "R": (_P, _P, 2, 2), "Rinv": (_P, _P, 2, 2), "cmu": (_P, _K, _K), "A": (_P, _K, _K),
                  "Beff": (_P, _K), "Bfill": (_P, _K), "B": (_P, _K), "C": (_P,), "Diff": (_P, _K, _K)}
        return np.ctypeslib.as_array(getattr(self, name)).reshape(shapes[name])

    def copy(self) -> "GpModel":
        m = GpModel()
        C.memmove(C.byref(m), C.byref(self), C.sizeof(GpModel))
        return m


class GpStats(C.Structure):
    _fields_ = [
        ("phi_max", C.c_double * _P), ("phi_min", C.c_double * _P), ("rel_change_phi", C.c_double * _P),
        ("mu_max", C.c_double * _K), ("mu_min", C.c_double * _K), ("rel_change_mu", C.c_double * _K),
        ("solute", C.c_double * _K), ("phase_fraction", C.c_double * _P), ("nonfinite", C.c_int64),
        ("energy_gradient", C.c_double), ("energy_potential", C.c_double), ("energy_chemical", C.c_double),
        ("grand_potential", C.c_double),
    ]
    ENERGIES = ("energy_gradient", "energy_potential", "energy_chemical", "grand_potential")


_lib = None

_SIGS = {
    "gp_input_read": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "gp_input_free": (None, [C.c_void_p]),
    "gp_input_get_long": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64)]),
    "gp_input_get_double": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]),
    "gp_input_name": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_size_t]),
    "gp_model_from_input": (C.c_int, [C.c_void_p, C.POINTER(GpModel)]),
    "gp_fill": (C.c_int, [C.c_void_p, C.POINTER(GpModel), C.c_void_p, C.c_void_p]),
    "gp_write_vtk": (C.c_int, [C.c_void_p, C.POINTER(GpModel), C.c_char_p, C.c_void_p, C.c_void_p]),
    "gp_write_vtk_t": (C.c_int, [C.c_void_p, C.POINTER(GpModel), C.c_char_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "gp_set_time_step": (C.c_int, [C.c_void_p, C.c_int64]),
    "gp_set_compensated": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_get_compensated": (C.c_int, [C.c_void_p]),
    "gp_read_vtk": (C.c_int, [C.c_void_p, C.POINTER(GpModel), C.c_char_p, C.c_void_p, C.c_void_p]),
    "gp_create": (C.c_int, [C.POINTER(GpModel), C.c_int, C.POINTER(C.c_void_p)]),
    "gp_destroy": (C.c_int, [C.c_void_p]),
    "gp_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gp_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gp_step": (C.c_int, [C.c_void_p, C.c_int64]),
    "gp_sync": (C.c_int, [C.c_void_p]),
    "gp_get_stats": (C.c_int, [C.c_void_p, C.POINTER(GpStats)]),
    "gp_download_dphi": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gp_stream": (C.c_void_p, [C.c_void_p]),
    "gp_launch_count": (C.c_int64, [C.c_void_p]),
    "gp_model_sizeof": (C.c_size_t, []),
    "gp_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "gp_batch_destroy": (C.c_int, [C.c_void_p]),
    "gp_batch_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gp_batch_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gp_batch_upload_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gp_batch_download_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gp_batch_upload_all": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gp_batch_download_all": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gp_batch_step": (C.c_int, [C.c_void_p, C.c_int64]),
    "gp_batch_sync": (C.c_int, [C.c_void_p]),
    "gp_batch_get_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(GpStats)]),
    "gp_batch_get_stats_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "gp_batch_stats_from_raw": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(GpStats)]),
    "gp_batch_set_tile": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gp_batch_set_narrowband": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_batch_set_grids": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gp_batch_prepare": (C.c_int, [C.c_void_p]),
    "gp_batch_set_block": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_batch_get_block": (C.c_int, [C.c_void_p]),
    "gp_batch_set_scan": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_batch_get_scan": (C.c_int, [C.c_void_p]),
    "gp_batch_set_depth": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_batch_state_device": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "gp_batch_state_changed": (C.c_int, [C.c_void_p]),
    "gp_batch_get_depth": (C.c_int, [C.c_void_p]),
    "gp_batch_set_compensated": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_batch_set_time_step": (C.c_int, [C.c_void_p, C.c_int64]),
    "gp_batch_get_compensated": (C.c_int, [C.c_void_p]),
    "gp_batch_test_lose_box": (C.c_int, [C.c_void_p]),
    "gp_batch_get_grids": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
    "gp_batch_lean_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64)]),
    "gp_batch_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_batch_kernel_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "gp_batch_autotune": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "gp_batch_stream": (C.c_void_p, [C.c_void_p]),
    "gp_batch_launch_count": (C.c_int64, [C.c_void_p]),
    "gp_batch_cells": (C.c_int64, [C.c_void_p]),
    "gp_last_error": (C.c_char_p, []),
    "gp_set_device": (C.c_int, [C.c_int]),
    "gp_smooth": (C.c_int, [C.c_void_p, C.c_int64]),
    "gp_state_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                  C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "gp_state_changed": (C.c_int, [C.c_void_p]),
    "gp_interface_y": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "gp_shift_y": (C.c_int, [C.c_void_p, C.c_int64]),
    "gp_adj_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "gp_adj_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                 C.c_void_p]),
    "gp_adj_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gp_adj_stored_states": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "gp_adj_destroy": (C.c_int, [C.c_void_p]),
}


def _out(a, shape):
    """A C-contiguous float64 output array of `shape`: `a` itself when given."""
    if a is None:
        return np.empty(shape)
    if a.dtype != np.float64 or a.shape != tuple(shape) or not a.flags.c_contiguous or not a.flags.writeable:
        raise ValueError(f"output array must be writeable C-contiguous float64 of shape {tuple(shape)}")
    return a


def lib():
    """Load libgp_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `make -C {HERE}` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.gp_model_sizeof() != C.sizeof(GpModel):
            raise ImportError("gp_model layout mismatch between binding and library")
        _lib = L
    return _lib


class GpError(RuntimeError):
    def __init__(self, what: str, rc: int):
        msg = lib().gp_last_error() or b""
        super().__init__(f"{what} failed ({rc}): {msg.decode(errors='replace')}")
        self.rc = rc


def _check(what, rc):
    if rc != GP_OK:
        raise GpError(what, rc)


def set_device(device: int):
    """The GPU the library's contexts and batches created next on this thread use
    (the library's CUDA runtime is its own: torch.cuda.set_device does not reach it)."""
    _check("gp_set_device", lib().gp_set_device(int(device)))


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data


class Input:
    """Parsed Input.in + Filling.in (reference semantics, C side)."""

    def __init__(self, input_in: str, filling_in: str | None = None):
        h = C.c_void_p()
        _check("gp_input_read", lib().gp_input_read(input_in.encode(), filling_in.encode() if filling_in else None,
                                                     C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().gp_input_free(self._h)
            self._h = None

    def get_long(self, key: str) -> int:
        v = C.c_int64()
        _check("gp_input_get_long(%s)" % key, lib().gp_input_get_long(self._h, key.encode(), C.byref(v)))
        return v.value

    def get_double(self, key: str) -> float:
        v = C.c_double()
        _check("gp_input_get_double(%s)" % key, lib().gp_input_get_double(self._h, key.encode(), C.byref(v)))
        return v.value

    def name(self, which: int, index: int) -> str:
        buf = C.create_string_buffer(GP_NAME_LEN)
        _check("gp_input_name", lib().gp_input_name(self._h, which, index, buf, GP_NAME_LEN))
        return buf.value.decode()

    def model(self) -> GpModel:
        m = GpModel()
        _check("gp_model_from_input", lib().gp_model_from_input(self._h, C.byref(m)))
        return m

    def fill(self, m: GpModel):
        phi = np.zeros((m.N, m.mesh_x, m.mesh_y))
        mu = np.zeros((m.K1, m.mesh_x, m.mesh_y))
        _check("gp_fill", lib().gp_fill(self._h, C.byref(m), _ptr(phi), _ptr(mu)))
        return phi, mu

    def write_vtk(self, m: GpModel, path: str, phi: np.ndarray, mu: np.ndarray, tstep: int = 0):
        """DATA/<out>_<t>.vtk as the reference writes it; tstep: the step the fields are after (the
        frozen gradient's temperature of a non-isothermal model)."""
        phi = np.ascontiguousarray(phi, dtype=np.float64)  # held: the C call reads them
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        _check("gp_write_vtk_t", lib().gp_write_vtk_t(self._h, C.byref(m), path.encode(), _ptr(phi), _ptr(mu),
                                                        int(tstep)))

    def read_vtk(self, m: GpModel, path: str):
        phi = np.zeros((m.N, m.mesh_x, m.mesh_y))
        mu = np.zeros((m.K1, m.mesh_x, m.mesh_y))
        _check("gp_read_vtk", lib().gp_read_vtk(self._h, C.byref(m), path.encode(), _ptr(phi), _ptr(mu)))
        return phi, mu


class Context:
    """One simulation instance resident on the current CUDA device."""

    def __init__(self, model: GpModel, precision: int = GP_FP64):
        h = C.c_void_p()
        self.model = model.copy()
        _check("gp_create", lib().gp_create(C.byref(self.model), precision, C.byref(h)))
        self._h = h
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            lib().gp_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, phi: np.ndarray, mu: np.ndarray):
        phi = np.ascontiguousarray(phi, dtype=np.float64)  # held: the C call reads them
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        _check("gp_upload", lib().gp_upload(self._h, _ptr(phi), _ptr(mu)))

    def download(self, phi: np.ndarray | None = None, mu: np.ndarray | None = None):
        """The state as float64 arrays (into phi / mu when given)."""
        m = self.model
        phi = _out(phi, (m.N, m.mesh_x, m.mesh_y))
        mu = _out(mu, (m.K1, m.mesh_x, m.mesh_y))
        _check("gp_download", lib().gp_download(self._h, _ptr(phi), _ptr(mu)))
        return phi, mu

    def download_dphi(self):
        m = self.model
        d = np.empty((m.N, m.mesh_x + 2, m.mesh_y + 2))
        _check("gp_download_dphi", lib().gp_download_dphi(self._h, _ptr(d)))
        return d

    def step(self, nsteps: int = 1):
        _check("gp_step", lib().gp_step(self._h, int(nsteps)))

    def smooth(self, nsteps: int):
        """nsteps smoothing pre-steps (NSMOOTH - 1 in the reference's main)."""
        _check("gp_smooth", lib().gp_smooth(self._h, int(nsteps)))

    def set_time_step(self, t: int):
        """The step count the frozen temperature gradient is evaluated at."""
        _check("gp_set_time_step", lib().gp_set_time_step(self._h, int(t)))

    def set_compensated(self, on: bool):
        """FP32 only: compensated (error-free transform) accumulation of the updates."""
        _check("gp_set_compensated", lib().gp_set_compensated(self._h, int(bool(on))))

    def compensated(self) -> bool:
        return bool(lib().gp_get_compensated(self._h))

    def device_state(self):
        """(phi, mu) torch views [planes, mesh_x, pitch] of the current device
        buffers (valid until the next step); call state_changed() after writing."""
        ph, mu_, pitch, plane, es = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64(), C.c_int()
        _check("gp_state_device", lib().gp_state_device(self._h, C.byref(ph), C.byref(mu_), C.byref(pitch),
                                                          C.byref(plane), C.byref(es)))
        return _device_views(self.model, ph.value, mu_.value, pitch.value, plane.value, es.value)

    def state_changed(self):
        _check("gp_state_changed", lib().gp_state_changed(self._h))

    def interface_y(self) -> int:
        """Highest upward liquid crossing, ghost-padded row index (check_SHIFT)."""
        v = C.c_int64()
        _check("gp_interface_y", lib().gp_interface_y(self._h, C.byref(v)))
        return v.value

    def shift_y(self, d: int):
        """Move the window d rows along +y (apply_shiftY)."""
        _check("gp_shift_y", lib().gp_shift_y(self._h, int(d)))

    def sync(self):
        _check("gp_sync", lib().gp_sync(self._h))

    def stats(self, allow_nonfinite: bool = False) -> dict:
        st = GpStats()
        rc = lib().gp_get_stats(self._h, C.byref(st))
        if rc != GP_OK and not (allow_nonfinite and rc == GP_E_NONFINITE):
            raise GpError("gp_get_stats", rc)
        return _stats_dict(st, self.model.N, self.model.K1)

    @property
    def stream(self) -> int:
        return lib().gp_stream(self._h) or 0

    @property
    def launches(self) -> int:
        return lib().gp_launch_count(self._h)


def _device_views(model, ph: int, mu: int, pitch: int, plane: int, esize: int):
    """torch views [planes, mesh_x, pitch] of a state's phi and mu device buffers."""
    import torch
    typestr = "<f8" if esize == 8 else "<f4"
    mx = int(model.mesh_x)

    class _View:
        def __init__(self, ptr, planes):
            self.__cuda_array_interface__ = {"shape": (planes, mx, pitch), "typestr": typestr,
                                             "data": (ptr, False), "version": 3,
                                             "strides": (plane * esize, pitch * esize, esize)}
    return (torch.as_tensor(_View(ph, int(model.N)), device="cuda"),
            torch.as_tensor(_View(mu, int(model.K1)), device="cuda"))


def _stats_dict(st: GpStats, N: int, K1: int) -> dict:
    out = {n: np.array(getattr(st, n)[: (N if ("phi" in n or "phase" in n) else K1)])
           for n, _ in GpStats._fields_ if n != "nonfinite" and n not in GpStats.ENERGIES}
    out["nonfinite"] = st.nonfinite
    for n in GpStats.ENERGIES:
        out[n] = float(getattr(st, n))
    out["free_energy"] = out["energy_gradient"] + out["energy_potential"] + out["energy_chemical"]
    return out


class Batch:
    """Many independent instances stepped together (FP32 chosen form)."""

    def __init__(self, models):
        self.models = [m.copy() for m in models]
        arr = (GpModel * len(models))(*self.models)
        h = C.c_void_p()
        _check("gp_batch_create", lib().gp_batch_create(C.cast(arr, C.c_void_p), len(models), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().gp_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.models)

    def upload(self, i: int, phi: np.ndarray, mu: np.ndarray, wait: bool = True):
        """Instance i's state from float64 arrays.  wait=False queues the copy on the batch's
        stream and returns (the arrays must then be C-contiguous float64, ideally page-locked,
        and stay untouched until sync())."""
        if not wait:
            for a in (phi, mu):
                if a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError("upload(wait=False) needs C-contiguous float64 arrays")
            _check("gp_batch_upload_async", lib().gp_batch_upload_async(self._h, i, _ptr(phi), _ptr(mu)))
            return
        phi = np.ascontiguousarray(phi, dtype=np.float64)  # held: the C call reads them
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        _check("gp_batch_upload", lib().gp_batch_upload(self._h, i, _ptr(phi), _ptr(mu)))

    def download(self, i: int, phi: np.ndarray | None = None, mu: np.ndarray | None = None, wait: bool = True):
        """Instance i's state as float64 arrays (into phi / mu when given: C-contiguous
        float64 of the instance's shapes, e.g. views of pinned host memory).  wait=False
        queues the copy on the batch's stream: the arrays hold the state after sync()."""
        m = self.models[i]
        phi = _out(phi, (m.N, m.mesh_x, m.mesh_y))
        mu = _out(mu, (m.K1, m.mesh_x, m.mesh_y))
        if not wait:
            _check("gp_batch_download_async", lib().gp_batch_download_async(self._h, i, _ptr(phi), _ptr(mu)))
        else:
            _check("gp_batch_download", lib().gp_batch_download(self._h, i, _ptr(phi), _ptr(mu)))
        return phi, mu

    def upload_all(self, fields):
        """Every instance's state from [(phi, mu), ...], queued (sync() waits): C-contiguous
        float64 arrays, read in place by one conversion launch when page-locked."""
        for a in (x for f in fields for x in f):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("upload_all needs C-contiguous float64 arrays")
        ptrs = (C.c_void_p * len(fields))
        _check("gp_batch_upload_all", lib().gp_batch_upload_all(
            self._h, ptrs(*[f[0].ctypes.data for f in fields]), ptrs(*[f[1].ctypes.data for f in fields])))

    def download_all(self, fields):
        """Every instance's state into [(phi, mu), ...] (writeable C-contiguous float64 arrays of the
        instances' shapes), queued: the arrays hold it after sync()."""
        for i, (p, u) in enumerate(fields):
            m = self.models[i]
            _out(p, (m.N, m.mesh_x, m.mesh_y))
            _out(u, (m.K1, m.mesh_x, m.mesh_y))
        ptrs = (C.c_void_p * len(fields))
        _check("gp_batch_download_all", lib().gp_batch_download_all(
            self._h, ptrs(*[f[0].ctypes.data for f in fields]), ptrs(*[f[1].ctypes.data for f in fields])))

    def step(self, nsteps: int = 1):
        _check("gp_batch_step", lib().gp_batch_step(self._h, int(nsteps)))

    def sync(self):
        _check("gp_batch_sync", lib().gp_batch_sync(self._h))

    def stats(self, i: int, allow_nonfinite: bool = False) -> dict:
        st = GpStats()
        rc = lib().gp_batch_get_stats(self._h, i, C.byref(st))
        if rc != GP_OK and not (allow_nonfinite and rc == GP_E_NONFINITE):
            raise GpError("gp_batch_get_stats", rc)
        return _stats_dict(st, self.models[i].N, self.models[i].K1)

    def stats_async(self, i: int, raw: np.ndarray):
        """Queue instance i's statistics read-back into `raw` (page-locked, C-contiguous float64,
        GP_STAT_VALUES entries) without waiting; after sync(), stats_from_raw(i, raw) decodes it."""
        if raw.dtype != np.float64 or raw.size < GP_STAT_VALUES or not raw.flags.c_contiguous:
            raise ValueError(f"raw must be a C-contiguous float64 array of at least {GP_STAT_VALUES} values")
        _check("gp_batch_get_stats_async", lib().gp_batch_get_stats_async(self._h, i, raw.ctypes.data))

    def stats_from_raw(self, i: int, raw: np.ndarray, allow_nonfinite: bool = False) -> dict:
        st = GpStats()
        v = np.ascontiguousarray(raw, dtype=np.float64)
        if v.size < GP_STAT_VALUES:
            raise ValueError(f"raw must hold {GP_STAT_VALUES} values")
        rc = lib().gp_batch_stats_from_raw(self._h, i, v.ctypes.data, C.byref(st))
        if rc != GP_OK and not (allow_nonfinite and rc == GP_E_NONFINITE):
            raise GpError("gp_batch_stats_from_raw", rc)
        return _stats_dict(st, self.models[i].N, self.models[i].K1)

    def set_tile(self, tx: int, ty: int):
        _check("gp_batch_set_tile", lib().gp_batch_set_tile(self._h, tx, ty))

    def set_narrowband(self, on: bool):
        _check("gp_batch_set_narrowband", lib().gp_batch_set_narrowband(self._h, 1 if on else 0))

    def set_block(self, threads: int):
        """Threads per full-kernel block: 256, or 512 for binary alloys."""
        _check("gp_batch_set_block", lib().gp_batch_set_block(self._h, threads))

    def block(self) -> int:
        return lib().gp_batch_get_block(self._h)

    def set_scan(self, on: bool):
        """Full-kernel blocks find their own interface tiles (True) or take them from the list."""
        _check("gp_batch_set_scan", lib().gp_batch_set_scan(self._h, 1 if on else 0))

    def scan(self) -> bool:
        return bool(lib().gp_batch_get_scan(self._h))

    def device_state(self, i: int):
        """(phi, mu) torch views [planes, mesh_x, pitch] of instance i's current
        device buffers (valid until the next step); call state_changed() after writing."""
        ph, mu_, pitch, plane, es = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64(), C.c_int()
        _check("gp_batch_state_device", lib().gp_batch_state_device(self._h, i, C.byref(ph), C.byref(mu_),
                                                                      C.byref(pitch), C.byref(plane), C.byref(es)))
        return _device_views(self.models[i], ph.value, mu_.value, pitch.value, plane.value, es.value)

    def state_changed(self):
        _check("gp_batch_state_changed", lib().gp_batch_state_changed(self._h))

    def set_depth(self, depth: int):
        """Temporal blocking: 1 (single steps) or 2 (blocked pairs; narrow band in list mode)."""
        _check("gp_batch_set_depth", lib().gp_batch_set_depth(self._h, depth))

    def depth(self) -> int:
        return lib().gp_batch_get_depth(self._h)

    def set_time_step(self, t: int):
        """The step count the frozen temperature gradient is evaluated at (steps taken)."""
        _check("gp_batch_set_time_step", lib().gp_batch_set_time_step(self._h, int(t)))

    def set_compensated(self, on: bool):
        """Compensated (error-free transform) accumulation of the FP32 updates."""
        _check("gp_batch_set_compensated", lib().gp_batch_set_compensated(self._h, int(bool(on))))

    def compensated(self) -> bool:
        return bool(lib().gp_batch_get_compensated(self._h))

    def prepare(self):
        """Capture the step graphs now (no step is taken)."""
        _check("gp_batch_prepare", lib().gp_batch_prepare(self._h))

    def set_grids(self, lean_per_sm: int = 0, general_per_sm: int = 0):
        """Blocks per SM of the lean and full persistent grids (0: as many as fit)."""
        _check("gp_batch_set_grids", lib().gp_batch_set_grids(self._h, lean_per_sm, general_per_sm))

    def grids(self):
        """(lean blocks per SM, full blocks per SM, lean occupancy, full occupancy)."""
        v = [C.c_int() for _ in range(4)]
        _check("gp_batch_get_grids", lib().gp_batch_get_grids(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def lean_tiles(self):
        """(tiles the next step updates with the lean kernel, all tiles)."""
        return self.lean_stats()[:2]

    def lean_stats(self):
        """(lean tiles of the next step, all tiles, interior cells of the lean tiles)."""
        lean, total, cells = C.c_int64(), C.c_int64(), C.c_int64()
        _check("gp_batch_lean_tiles",
               lib().gp_batch_lean_tiles(self._h, C.byref(lean), C.byref(total), C.byref(cells)))
        return lean.value, total.value, cells.value

    def set_timing(self, on: bool):
        """Per-kernel CUDA-event timing of every step (steps launch directly while on)."""
        _check("gp_batch_set_timing", lib().gp_batch_set_timing(self._h, 1 if on else 0))

    def kernel_ms(self):
        """Mean ms per step of the lean, list and full kernels since timing was switched on."""
        ms = (C.c_double * 3)()
        n = C.c_int64()
        _check("gp_batch_kernel_ms", lib().gp_batch_kernel_ms(self._h, ms, C.byref(n)))
        return {"lean": ms[0], "list": ms[1], "general": ms[2], "steps": n.value}

    def autotune(self, cache_path: str | None = None):
        tx, ty = C.c_int(), C.c_int()
        _check("gp_batch_autotune", lib().gp_batch_autotune(self._h, cache_path.encode() if cache_path else None,
                                                            C.byref(tx), C.byref(ty)))
        return tx.value, ty.value

    @property
    def stream(self) -> int:
        return lib().gp_batch_stream(self._h) or 0

    @property
    def launches(self) -> int:
        return lib().gp_batch_launch_count(self._h)

    @property
    def cells(self) -> int:
        return lib().gp_batch_cells(self._h)


def load_case(case):
    """Input files of a configs.Case -> (model, phi, mu) through the C parser."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        ip, fp = case.write(d)
        inp = Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    return m, phi, mu
