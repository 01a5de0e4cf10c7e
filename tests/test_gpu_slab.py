"""One grid split into x-slabs on the GPU: the slabs of one process (sharing
the GPU) step through the C ABI contexts and exchange halo rows with device
copies every `depth` steps; owned rows equal the single-grid run bit for bit,
FP64 and FP32, Neumann and periodic x."""
import tempfile

import numpy as np
import pytest

from conftest import load_golden, write_inputs
import microsim_b200 as mb
from microsim_b200 import configs, slab as S

pytestmark = pytest.mark.gpu


def _case(name):
    if name == "corner_96x64":
        return mb.load_case(configs.binary_case(96, 64, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05,
                                                tau=1.7776, seed=(0, 0, 8.0)))
    g = load_golden(name)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    return m, phi, mu


@pytest.mark.parametrize("precision", [mb.GP_FP64, mb.GP_FP32])
@pytest.mark.parametrize("name,world,depth", [("iso_obst_bin", 2, 2), ("aniso_obst_bin_per", 2, 1),
                                              ("corner_96x64", 3, 3)])
def test_slabs_equal_the_single_grid(name, world, depth, precision):
    m, phi, mu = _case(name)
    steps = 24
    with mb.Context(m, precision) as c:
        c.upload(phi, mu)
        c.step(steps)
        gp, gu = c.download()
    mx, bc_x = int(m.mesh_x), int(m.bc_phi[0])
    slabs, copies = S.plan(mx, world, bc_x, depth)
    ctxs = []
    try:
        for s in slabs:
            rows = [S.gmap(g, mx, bc_x) if (g < 0 or g >= mx) else g for g in range(s.lo, s.hi)]
            c = mb.Context(S.local_model(m, s), precision)
            c.upload(np.ascontiguousarray(phi[:, rows]), np.ascontiguousarray(mu[:, rows]))
            ctxs.append(c)
        for _ in range(steps // depth):
            for c in ctxs:
                c.step(depth)
            S.exchange_local(ctxs, copies)
        for s, c in zip(slabs, ctxs):
            p, u = c.download()
            own = slice(s.own_lo - s.lo, s.own_hi - s.lo)
            assert np.array_equal(p[:, own], gp[:, s.own_lo:s.own_hi]), (s.rank, np.abs(p[:, own] - gp[:, s.own_lo:s.own_hi]).max())
            assert np.array_equal(u[:, own], gu[:, s.own_lo:s.own_hi])
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("depth_blocking", [1, 2])
def test_slabs_as_instances_of_one_fp32_batch(depth_blocking):
    """The slabs as the instances of one FP32 batch (narrow band, temporal blocking of
    the given depth inside the batch), halo rows exchanged on the batch's stream every
    `depth` steps with no host wait: owned rows equal the single-grid FP32 run."""
    m, phi, mu = _case("corner_96x64")
    steps, depth, world = 24, 2, 3
    with mb.Context(m, mb.GP_FP32) as c:
        c.upload(phi, mu)
        c.step(steps)
        gp, gu = c.download()
    mx, bc_x = int(m.mesh_x), int(m.bc_phi[0])
    slabs, copies = S.plan(mx, world, bc_x, depth)
    with mb.Batch([S.local_model(m, s) for s in slabs]) as b:
        b.set_depth(depth_blocking)
        for i, s in enumerate(slabs):
            rows = [S.gmap(g, mx, bc_x) if (g < 0 or g >= mx) else g for g in range(s.lo, s.hi)]
            b.upload(i, np.ascontiguousarray(phi[:, rows]), np.ascontiguousarray(mu[:, rows]))
        for _ in range(steps // depth):
            b.step(depth)
            S.exchange_batch_local(b, copies)
        for i, s in enumerate(slabs):
            p, u = b.download(i)
            own = slice(s.own_lo - s.lo, s.own_hi - s.lo)
            assert np.array_equal(p[:, own], gp[:, s.own_lo:s.own_hi]), (s.rank, np.abs(p[:, own] - gp[:, s.own_lo:s.own_hi]).max())
            assert np.array_equal(u[:, own], gu[:, s.own_lo:s.own_hi])
