"""Plain form (FP64) on the GPU through the C ABI, against the reference.

The bar is bit-exact: the fixtures in tests/golden were written by the
reference serial solver compiled from its own sources, and the FP64 kernels
keep its operation order with no FMA contraction.  Longer runs compare with the
oracle restatement (itself pinned bit-exact to the reference by
tests/test_oracle_golden.py) and, for the 200x200 x 10,000-step workload, with
per-row SHA-256 digests of the reference's final state.
"""
import tempfile

import numpy as np
import pytest

from conftest import (golden_cases, interior, load_golden, long_cases, oracle_model, presmooth, row_digests,
                      write_inputs)
import microsim_b200 as mb
from microsim_b200 import configs
from oracle import gp_oracle as O

pytestmark = pytest.mark.gpu


def _setup(g):
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    return m, phi, mu


@pytest.mark.parametrize("case", golden_cases())
def test_dphi_ring_bitexact(case):
    g = load_golden(case)
    m, phi, mu = _setup(g)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        presmooth(ctx, g)
        ctx.step(1)
        d = ctx.download_dphi()
    ref = g["dphi_1"][:, 2:-2, 2:-2]
    assert np.array_equal(d, ref), f"max |diff| {np.abs(d - ref).max()}"


@pytest.mark.parametrize("case", [c for c in golden_cases() if "nsmooth" in load_golden(c)])
@pytest.mark.parametrize("precision", [mb.GP_FP64, mb.GP_FP32])
def test_smoothing_pre_steps_bitexact(case, precision):
    """NSMOOTH - 1 pre-steps equal the reference's.  An FP32 context runs them in
    FP64 from its FP32-stored state: within 1e-6 of the reference."""
    g = load_golden(case)
    m, phi, mu = _setup(g)
    with mb.Context(m, precision) as ctx:
        ctx.upload(phi, mu)
        ctx.smooth(int(g["nsmooth"]) - 1)
        p, u = ctx.download()
    rp, ru = interior(g["phi_smoothed"]), interior(g["mu_smoothed"])
    if precision == mb.GP_FP64:
        assert np.array_equal(p, rp) and np.array_equal(u, ru)
    else:
        assert np.abs(p - rp).max() <= 1e-6 and np.abs(u - ru).max() <= 1e-6


@pytest.mark.parametrize("case", [c for c in golden_cases() if "shifts" not in load_golden(c)])
def test_states_bitexact(case):
    g = load_golden(case)
    m, phi, mu = _setup(g)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        presmooth(ctx, g)
        done = 0
        for t in g["dump_steps"]:
            ctx.step(int(t) - done)
            done = int(t)
            p, u = ctx.download()
            assert np.array_equal(p, interior(g[f"phi_{t}"])), \
                f"phi after {t}: max |diff| {np.abs(p - interior(g[f'phi_{t}'])).max()}"
            assert np.array_equal(u, interior(g[f"mu_{t}"])), \
                f"mu after {t}: max |diff| {np.abs(u - interior(g[f'mu_{t}'])).max()}"


def _oracle_run(case, steps):
    """Oracle from the product's constants (those are pinned to the reference's)."""
    with tempfile.TemporaryDirectory() as d:
        ip, fp = case.write(d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    op, om_ = _oracle_from(m, phi, mu, steps)
    return m, phi, mu, op, om_


def _oracle_from(m, phi, mu, steps):
    """The oracle's state after `steps` steps from the interior fields phi, mu."""
    om = O.OracleModel(
        N=m.N, K1=m.K1, mesh_x=m.mesh_x, mesh_y=m.mesh_y, dx=m.dx, dy=m.dy, dt=m.dt, epsilon=m.epsilon, tau=m.tau,
        T=m.T, Teq=m.Teq, obstacle=m.obstacle, anisotropy=m.anisotropy, binary=int(m.mu_solver == mb.GP_MU_BINARY),
        ternary=int(m.mu_solver == mb.GP_MU_TERNARY), dilute=int(m.mu_solver == mb.GP_MU_DILUTE),
        bc_phi=tuple(m.bc_phi), bc_mu=tuple(m.bc_mu),
        Gamma=m.arr("Gamma")[:m.N, :m.N], tau_ab=m.arr("tau_ab")[:m.N, :m.N], cmu=m.arr("cmu")[:m.N, :m.K1, :m.K1],
        A=m.arr("A")[:m.N, :m.K1, :m.K1], Beq=m.arr("Beff")[:m.N, :m.K1], dBbdT=np.zeros((m.N, m.K1)),
        B=m.arr("B")[:m.N, :m.K1], C=m.arr("C")[:m.N], Diff=m.arr("Diff")[:m.N, :m.K1, :m.K1],
        dab=m.arr("dab")[:m.N, :m.N],
        R=np.pad(m.arr("R")[:m.N, :m.N], ((0, 0), (0, 0), (0, 1), (0, 1))),
        Rinv=np.pad(m.arr("Rinv")[:m.N, :m.N], ((0, 0), (0, 0), (0, 1), (0, 1))),
        Gamma_abc=m.arr("Gamma_abc")[:m.N, :m.N, :m.N])
    gp = np.zeros((m.N, m.mesh_x + 6, m.mesh_y + 6))
    gm = np.zeros((m.K1, m.mesh_x + 6, m.mesh_y + 6))
    gp[:, 3:-3, 3:-3], gm[:, 3:-3, 3:-3] = phi, mu
    O.apply_bc(om, gp, gm)
    O.step(om, gp, gm, steps)
    return interior(gp), interior(gm)


LONG = {
    "aniso_dendrite_corner": (configs.binary_case(64, 48, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05,
                                                  tau=1.7776, seed=(0, 0, 8.0), steps=600), 600),
    "aniso_rot_periodic_well": (configs.binary_case(48, 40, gap=1.0, supersat=0.45, eps=3.0, delta=0.05,
                                                    theta=33.0, dt=0.05, tau=1.3332, function_w=2,
                                                    seed=(20, 20, 7.0), bc=(3, 3, 3, 3), steps=400), 400),
    "c3_small": (configs.c3(steps=200, mesh=56, nseeds=8, rng_seed=5), 200),
}


@pytest.mark.parametrize("name", sorted(LONG))
def test_long_runs_bitexact_vs_oracle(name):
    case, steps = LONG[name]
    m, phi, mu, op, om_ = _oracle_run(case, steps)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        ctx.step(steps)
        p, u = ctx.download()
    assert np.array_equal(p, op), f"phi max |diff| {np.abs(p - op).max()}"
    assert np.array_equal(u, om_), f"mu max |diff| {np.abs(u - om_).max()}"


def test_graph_replayed_steps_equal_single_steps():
    """Isothermal FP64 runs of eight or more steps replay a captured graph from
    either buffer; the states equal those of steps launched one at a time, bit
    for bit, whatever the split of the step counts."""
    case, _ = LONG["aniso_dendrite_corner"]
    with tempfile.TemporaryDirectory() as d:
        ip, fp = case.write(d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    with mb.Context(m, mb.GP_FP64) as one, mb.Context(m, mb.GP_FP64) as many:
        one.upload(phi, mu)
        many.upload(phi, mu)
        done = 0
        for n in (8, 1, 8, 17, 3, 16, 9):  # graphs from buffer 0 and from buffer 1, with remainders
            for _ in range(n):
                one.step(1)
            many.step(n)
            done += n
            p1, u1 = one.download()
            pn, un = many.download()
            assert np.array_equal(p1, pn) and np.array_equal(u1, un), (done, n)


def test_flat_blocks_outside_the_simplex_take_the_full_evaluation():
    """The kernels skip the arithmetic of cells whose 3x3 phi block is one value per phase in
    [0, 1].  Flat patches just outside that range (a phase slightly negative, whose projection
    still changes Delta-phi, and one slightly above one) and a flat patch inside the interface
    range (0.5 / 0.5) step bit-exactly like the oracle."""
    case = configs.binary_case(40, 36, gap=1.0, supersat=0.5, eps=2.0, delta=0.02, dt=0.05, tau=0.9,
                               seed=(10, 10, 5.0), steps=20)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = case.write(d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    phi = phi.copy()
    phi[0, 24:34, 4:14], phi[1, 24:34, 4:14] = -1e-3, 1.0 + 1e-3
    phi[0, 4:14, 22:32], phi[1, 4:14, 22:32] = 0.5, 0.5
    phi[0, 24:34, 22:32], phi[1, 24:34, 22:32] = 1.0 + 2e-3, -2e-3
    op, om_ = _oracle_from(m, phi, mu, 20)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        for n in (1, 19):  # one direct step, then a graph replay and direct steps
            ctx.step(n)
        p, u = ctx.download()
    assert np.array_equal(p, op), f"phi max |diff| {np.abs(p - op).max()}"
    assert np.array_equal(u, om_), f"mu max |diff| {np.abs(u - om_).max()}"


RAGGED = [(4, 4, (1, 1, 1, 1)), (5, 7, (3, 3, 3, 3)), (4, 37, (1, 1, 3, 3)), (33, 5, (3, 3, 1, 1)),
          (6, 6, (1, 1, 1, 1))]


@pytest.mark.parametrize("mx,my,bc", RAGGED)
def test_smallest_and_ragged_grids(mx, my, bc):
    """The smallest grids the step takes (4 cells on an axis) and ragged ones, Neumann and periodic:
    FP64 bit-exact to the oracle, FP32 within its tolerance, and a FP32 batch of all of them
    (partial tiles only, the narrow band on) equal to FP32 contexts bit for bit."""
    case = configs.binary_case(mx, my, gap=1.0, supersat=0.5, eps=2.0, delta=0.02, dt=0.05, tau=0.9,
                               seed=(mx // 2, my // 2, min(mx, my) / 3.0), bc=bc, steps=50)
    m, phi, mu, op, om_ = _oracle_run(case, 50)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        ctx.step(50)
        p, u = ctx.download()
    assert np.array_equal(p, op) and np.array_equal(u, om_)
    with mb.Context(m, mb.GP_FP32) as ctx:
        ctx.upload(phi, mu)
        ctx.step(50)
        p32, u32 = ctx.download()
    assert np.abs(p32 - p).max() <= 1e-4 and np.abs(u32 - u).max() <= 1e-3


def test_ragged_grids_in_one_batch():
    loaded = [mb.load_case(configs.binary_case(mx, my, gap=1.0, supersat=0.5, eps=2.0, delta=0.02, dt=0.05,
                                               tau=0.9, seed=(mx // 2, my // 2, min(mx, my) / 3.0), bc=bc,
                                               steps=50)) for mx, my, bc in RAGGED]
    ref = []
    for m, phi, mu in loaded:
        with mb.Context(m, mb.GP_FP32) as ctx:
            ctx.upload(phi, mu)
            ctx.step(50)
            ref.append(ctx.download())
    with mb.Batch([m for m, _, _ in loaded]) as b:
        for i, (_, phi, mu) in enumerate(loaded):
            b.upload(i, phi, mu)
        b.step(50)
        for i, (p0, u0) in enumerate(ref):
            p1, u1 = b.download(i)
            assert np.array_equal(p1, p0) and np.array_equal(u1, u0), i


def test_grids_below_four_cells_are_refused():
    case = configs.binary_case(3, 12, gap=1.0, supersat=0.5, eps=2.0, dt=0.05, tau=0.9, seed=(1, 6, 1.0), steps=5)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = case.write(d)
        with pytest.raises(mb.GpError):  # by the input reader or by the context
            mb.Context(mb.Input(ip, fp).model(), mb.GP_FP64)


@pytest.mark.parametrize("name", long_cases())
def test_config1_full_run_matches_reference(name):
    """200x200, 10,000 steps: every row of the final state equals the reference's."""
    g = dict(np.load(f"{__import__('conftest').GOLDEN}/{name}.long.npz"))
    m, phi, mu = _setup(g)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        ctx.step(int(g["steps"]))
        p, u = ctx.download()
    dig = row_digests(p, u)
    bad = np.nonzero(dig != g["row_sha256"])[0]
    sums = np.concatenate([p, u]).sum(axis=(1, 2))
    assert bad.size == 0, f"{bad.size} rows differ (first {bad[:5]}); plane sums {sums} vs {g['plane_sums']}"


def test_roundtrip_and_zero_steps():
    g = load_golden("three_phase_eutectic")
    m, phi, mu = _setup(g)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        ctx.step(0)
        p, u = ctx.download()
    assert np.array_equal(p, phi) and np.array_equal(u, mu)


def test_stats_against_host():
    g = load_golden("iso_obst_bin")
    m, phi, mu = _setup(g)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        ctx.step(5)
        p0, u0 = ctx.download()
        ctx.step(1)
        p1, u1 = ctx.download()
        st = ctx.stats()
    assert st["nonfinite"] == 0
    np.testing.assert_allclose(st["rel_change_phi"], ((p1 - p0) ** 2).sum(axis=(1, 2)), rtol=1e-12)
    np.testing.assert_allclose(st["rel_change_mu"], ((u1 - u0) ** 2).sum(axis=(1, 2)), rtol=1e-12)
    np.testing.assert_allclose(st["phase_fraction"], p1.sum(axis=(1, 2)), rtol=1e-12)
    assert np.all(st["phi_max"] >= p1.max(axis=(1, 2))) and np.all(st["phi_min"] <= p1.min(axis=(1, 2)))
    # solute: sum over cells of sum_a c_a(mu) h_a(phi)
    cmu, beff = m.arr("cmu")[:2, 0, 0], m.arr("Beff")[:2, 0]
    h0 = 3 * p1[0] ** 2 - 2 * p1[0] ** 3
    h1 = 3 * p1[1] ** 2 - 2 * p1[1] ** 3
    sol = (cmu[0] * (u1[0] - beff[0]) * h0 + cmu[1] * (u1[0] - beff[1]) * h1).sum()
    np.testing.assert_allclose(st["solute"][0], sol, rtol=1e-12)


def test_nan_watchdog():
    g = load_golden("iso_obst_bin")
    m, phi, mu = _setup(g)
    mu = mu.copy()
    mu[0, 3, 4] = np.nan
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        st = ctx.stats(allow_nonfinite=True)
        assert st["nonfinite"] >= 1
        with pytest.raises(mb.GpError) as e:
            ctx.stats()
        assert e.value.rc == mb.GP_E_NONFINITE


def test_create_rejects_bad_models():
    g = load_golden("iso_obst_bin")
    m, _, _ = _setup(g)
    bad = m.copy()
    bad.N = 9
    with pytest.raises(mb.GpError):
        mb.Context(bad, mb.GP_FP64)
    bad = m.copy()
    bad.bc_phi[0] = 0
    with pytest.raises(mb.GpError):
        mb.Context(bad, mb.GP_FP64)


def test_moving_frame_against_reference():
    """Shift = 1: the interface row found every 100 steps, the accumulated
    offset and the states equal the reference's, bit for bit (the phase-field
    half step after a shift reads the shifted ghost rows, as the reference's)."""
    g = load_golden("shift_planar")
    m, phi, mu = _setup(g)
    shiftj = 20
    offset, done, k = 0, 0, 0
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        for t in g["dump_steps"]:
            t = int(t)
            while done < t:
                nxt = min(t, (done // 100 + 1) * 100)
                ctx.step(nxt - done)
                done = nxt
                if done % 100 == 0:
                    pos = ctx.interface_y()
                    assert pos == g["shifts"][k][1], (done, pos, g["shifts"][k])
                    if pos > shiftj:
                        ctx.shift_y(pos - shiftj)
                        offset += pos - shiftj
                    assert offset == g["shifts"][k][2]
                    k += 1
            p, u = ctx.download()
            rp, ru = interior(g[f"phi_{t}"]), interior(g[f"mu_{t}"])
            assert np.array_equal(p, rp) and np.array_equal(u, ru), \
                (t, np.abs(p - rp).max(), np.abs(u - ru).max())
    assert k == len(g["shifts"])
