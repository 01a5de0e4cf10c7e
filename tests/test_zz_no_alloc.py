"""The allocation-free FP64 step, gp_step_f64_noalloc, through the C ABI.

Some callers own their device buffers and cannot allocate device memory (a
framework pool that owns the GPU, a fixed start-up memory budget).  For them
gp_step_f64_noalloc runs one plain step on buffers they pass in and keeps its
Delta-phi scratch in a fixed file-scope device array.  Here the test itself
holds the state buffers (torch tensors); the entry point allocates nothing.

Its results must equal the regular entry point's (gp_create/gp_step) exactly --
the plain form's tolerance everywhere in these tests is bit equality -- on two
calls in a row (the second call reuses the shared scratch array).  This file is
named to be collected last.
"""
import ctypes as C
import tempfile

import numpy as np
import pytest

from conftest import load_golden, write_inputs
import microsim_b200 as mb

pytestmark = pytest.mark.gpu


def _entry():
    f = mb.lib().gp_step_f64_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(mb.GpModel), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    return f


def _model(case):
    g = load_golden(case)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    return m, phi, mu


def _poison_scratch(f, m, dev, stream):
    """One call on a larger grid (480 x 480, within the fixed scratch for up to 4 phases) whose
    mu is NaN and whose phi is random, so every phase is active and the Delta-phi ring the call
    leaves in the shared scratch array is NaN over more than the following grid's extent.  The
    next call must rewrite every ring cell it reads, or NaN reaches its results."""
    import torch

    big = m.copy()
    big.mesh_x, big.mesh_y = 480, 480
    g = torch.Generator(device="cpu").manual_seed(7)
    P = torch.rand((m.N, 480, 480), generator=g, dtype=torch.float64).to(dev)
    U = torch.full((m.K1, 480, 480), float("nan"), dtype=torch.float64, device=dev)
    P2, U2 = torch.empty_like(P), torch.empty_like(U)
    rc = f(C.byref(big), P.data_ptr(), U.data_ptr(), P2.data_ptr(), U2.data_ptr(), 480, stream.cuda_stream)
    assert rc == mb.GP_OK, mb.lib().gp_last_error()
    torch.cuda.synchronize(dev)
    assert torch.isnan(P2).any()  # the poison reached the step (and so the ring)


@pytest.mark.parametrize("case,pitch_pad", [("aniso_obst_bin_per", 0), ("four_phase_ternary", 40),
                                            ("three_phase_eutectic", 7)])
def test_noalloc_matches_regular_step_twice(case, pitch_pad):
    import torch

    m, phi, mu = _model(case)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        ctx.step(1)
        want1 = ctx.download()
        ctx.step(1)
        want2 = ctx.download()

    mx, my = m.mesh_x, m.mesh_y
    pitch = my + pitch_pad
    dev = torch.device("cuda", torch.cuda.current_device())

    def dev_state(p, u):
        P = torch.zeros((m.N, mx, pitch), dtype=torch.float64, device=dev)
        U = torch.zeros((m.K1, mx, pitch), dtype=torch.float64, device=dev)
        P[:, :, :my] = torch.from_numpy(p)
        U[:, :, :my] = torch.from_numpy(u)
        return P, U

    pa, ua = dev_state(phi, mu)
    pb, ub = dev_state(np.zeros_like(phi), np.zeros_like(mu))
    stream = torch.cuda.current_stream(dev)
    f = _entry()
    _poison_scratch(f, m, dev, stream)
    torch.cuda.synchronize(dev)
    rc = f(C.byref(m), pa.data_ptr(), ua.data_ptr(), pb.data_ptr(), ub.data_ptr(), pitch, stream.cuda_stream)
    assert rc == mb.GP_OK, mb.lib().gp_last_error()
    rc = f(C.byref(m), pb.data_ptr(), ub.data_ptr(), pa.data_ptr(), ua.data_ptr(), pitch, stream.cuda_stream)
    assert rc == mb.GP_OK, mb.lib().gp_last_error()
    torch.cuda.synchronize(dev)
    got1 = (pb[:, :, :my].cpu().numpy(), ub[:, :, :my].cpu().numpy())
    got2 = (pa[:, :, :my].cpu().numpy(), ua[:, :, :my].cpu().numpy())
    for got, want in ((got1, want1), (got2, want2)):
        assert np.array_equal(got[0], want[0]), f"phi max |diff| {np.abs(got[0] - want[0]).max()}"
        assert np.array_equal(got[1], want[1]), f"mu max |diff| {np.abs(got[1] - want[1]).max()}"


def test_noalloc_rejects_grids_beyond_the_scratch_and_bad_buffers():
    import torch

    m, phi, mu = _model("aniso_obst_bin_per")
    f = _entry()
    dev = torch.device("cuda", torch.cuda.current_device())
    a = torch.zeros(8, dtype=torch.float64, device=dev)
    b = torch.zeros(8, dtype=torch.float64, device=dev)
    big = m.copy()
    big.mesh_x, big.mesh_y = 1024, 1024  # 2 * 1026 * 1056 doubles > 8 MiB: rejected before any launch
    rc = f(C.byref(big), a.data_ptr(), a.data_ptr() + 8, b.data_ptr(), b.data_ptr() + 8, 1024, None)
    assert rc == mb.GP_E_SIZE
    assert b"scratch" in mb.lib().gp_last_error()
    rc = f(C.byref(m), a.data_ptr(), a.data_ptr(), a.data_ptr(), b.data_ptr(), m.mesh_y, None)
    assert rc == mb.GP_E_ARG  # in place is refused
    # a partial overlap of an output with an input is refused too (phi_out starts inside phi)
    plane = m.mesh_x * m.mesh_y
    P = torch.zeros(4 * m.N * plane, dtype=torch.float64, device=dev)
    U = torch.zeros(2 * m.K1 * plane, dtype=torch.float64, device=dev)
    rc = f(C.byref(m), P.data_ptr(), U.data_ptr(), P.data_ptr() + 8 * plane, U.data_ptr() + 8 * m.K1 * plane,
           m.mesh_y, None)
    assert rc == mb.GP_E_ARG and b"overlaps" in mb.lib().gp_last_error()
    # mu_out overlapping phi (phi and mu packed into one buffer the wrong way) is refused
    rc = f(C.byref(m), P.data_ptr(), U.data_ptr(), P.data_ptr() + 8 * 2 * m.N * plane,
           P.data_ptr() + 8 * (m.N * plane - 1), m.mesh_y, None)
    assert rc == mb.GP_E_ARG and b"overlaps" in mb.lib().gp_last_error()
    # host memory is not a device buffer of the library's current device
    h = np.zeros(m.N * plane)
    rc = f(C.byref(m), h.ctypes.data, U.data_ptr(), P.data_ptr() + 8 * 2 * m.N * plane,
           U.data_ptr() + 8 * m.K1 * plane, m.mesh_y, None)
    assert rc == mb.GP_E_ARG and b"device memory" in mb.lib().gp_last_error()
