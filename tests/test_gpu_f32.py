"""Chosen form (FP32 storage and update, FP64 reductions) on the GPU.

Tolerances (max-abs over the interior) against the plain FP64 form, which is
itself bit-exact to the reference:
  * binary alloys, 400 steps:            phi <= 2e-5, mu <= 1e-4
  * four-phase ternary, 10 steps:        phi <= 1e-5, mu <= 2e-4
  * the reference fixtures after 40-60 steps: phi <= 1e-4 (2 phases),
    1e-3 (3 phases), 5e-3 (4 phases); mu ten times that
    (triple junctions amplify rounding differences into local branch flips of
     the simplex projection after ~100 steps; the solute mass still agrees)
  * solute mass (FP64 sum of sum_a c_a(mu) h_a(phi)): relative 1e-4
Determinism: every tile shape, a batch versus single contexts, and CUDA-graph
replay versus direct launches give identical bits.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, presmooth, write_inputs
import microsim_b200 as mb
from microsim_b200 import configs

pytestmark = pytest.mark.gpu

BINARY = {
    "iso": configs.binary_case(64, 48, gap=1.0, supersat=0.3, eps=4.0, dt=0.05, tau=1.7776, seed=(32, 24, 8.0)),
    "aniso_corner": configs.binary_case(64, 48, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05,
                                        tau=1.7776, seed=(0, 0, 8.0)),
    "aniso_rot_well_per": configs.binary_case(48, 40, gap=1.0, supersat=0.45, eps=3.0, delta=0.05, theta=33.0,
                                              dt=0.05, tau=1.3332, function_w=2, seed=(20, 20, 7.0),
                                              bc=(3, 3, 3, 3)),
}


def _pair(m, phi, mu, steps):
    with mb.Context(m, mb.GP_FP64) as c64, mb.Context(m, mb.GP_FP32) as c32:
        c64.upload(phi, mu)
        c32.upload(phi, mu)
        c64.step(steps)
        c32.step(steps)
        return c64.download(), c32.download(), c64.stats(), c32.stats()


@pytest.mark.parametrize("name", sorted(BINARY))
def test_binary_within_tolerance_of_fp64(name):
    m, phi, mu = mb.load_case(BINARY[name])
    (p64, u64), (p32, u32), s64, s32 = _pair(m, phi, mu, 400)
    assert np.abs(p32 - p64).max() <= 2e-5
    assert np.abs(u32 - u64).max() <= 1e-4
    np.testing.assert_allclose(s32["solute"], s64["solute"], rtol=1e-4)
    np.testing.assert_allclose(s32["phase_fraction"], s64["phase_fraction"], rtol=1e-4)


def test_four_phase_ternary_within_tolerance():
    m, phi, mu = mb.load_case(configs.c3(steps=200, mesh=56, nseeds=8, rng_seed=5))
    (p64, u64), (p32, u32), _, _ = _pair(m, phi, mu, 10)
    assert np.abs(p32 - p64).max() <= 1e-5
    assert np.abs(u32 - u64).max() <= 2e-4
    (p64, u64), (p32, u32), s64, s32 = _pair(m, phi, mu, 400)
    np.testing.assert_allclose(s32["solute"], s64["solute"], rtol=1e-4)


@pytest.mark.parametrize("case", [c for c in golden_cases()
                                  if c != "c1_literal_small" and "shifts" not in load_golden(c)])
def test_golden_cases_within_tolerance_of_reference(case):
    g = load_golden(case)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    t = int(g["dump_steps"][-1])
    with mb.Context(m, mb.GP_FP32) as c:
        c.upload(phi, mu)
        presmooth(c, g)
        c.step(t)
        p, u = c.download()
    tol = {2: 1e-4, 3: 1e-3}.get(m.N, 5e-3)  # triple junctions amplify FP32 rounding locally
    assert np.abs(p - interior(g[f"phi_{t}"])).max() <= tol
    assert np.abs(u - interior(g[f"mu_{t}"])).max() <= 10 * tol


def test_literal_config1_first_step():
    """The literal config-1 inputs are unstable (checkerboard); one step still matches."""
    g = load_golden("c1_literal_small")
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    with mb.Context(m, mb.GP_FP32) as c:
        c.upload(phi, mu)
        c.step(1)
        p, u = c.download()
    assert np.abs(p - interior(g["phi_1"])).max() <= 1e-5
    assert np.abs(u - interior(g["mu_1"])).max() <= 1e-5


def test_tile_shapes_batch_and_graph_are_bit_identical():
    m, phi, mu = mb.load_case(BINARY["aniso_corner"])
    res = {}
    for shape in [(16, 32), (8, 32), (32, 32), (16, 64)]:
        with mb.Batch([m]) as b:
            b.set_tile(*shape)
            b.upload(0, phi, mu)
            b.step(37)  # two graph replays of 16 steps + 5 direct launches
            res[shape] = b.download(0)
    ref = res[(16, 32)]
    for shape, v in res.items():
        assert np.array_equal(v[0], ref[0]) and np.array_equal(v[1], ref[1]), shape
    with mb.Context(m, mb.GP_FP32) as c:  # 37 direct launches
        c.upload(phi, mu)
        c.step(37)
        p, u = c.download()
    assert np.array_equal(p, ref[0]) and np.array_equal(u, ref[1])


def test_uneven_batch_equals_single_instances():
    cases = [configs.binary_case(40, 72, gap=1.0, supersat=0.5, eps=4.0, delta=0.03, dt=0.05, tau=1.7776,
                                 seed=(0, 0, 8.0)),
             configs.binary_case(96, 64, gap=1.0, supersat=0.35, eps=3.0, delta=0.01, theta=20.0, dt=0.05,
                                 tau=1.3332, seed=(40, 30, 9.0), bc=(3, 3, 1, 1)),
             configs.binary_case(33, 45, gap=1.0, supersat=0.6, eps=5.0, delta=0.05, dt=0.05, tau=2.222,
                                 function_w=2, seed=(10, 20, 6.0))]
    loaded = [mb.load_case(c) for c in cases]
    with mb.Batch([m for m, _, _ in loaded]) as b:
        for i, (_, p, u) in enumerate(loaded):
            b.upload(i, p, u)
        b.step(50)
        got = [b.download(i) for i in range(len(loaded))]
        st = [b.stats(i) for i in range(len(loaded))]
    for (m, p, u), (gp, gu), s in zip(loaded, got, st):
        with mb.Context(m, mb.GP_FP32) as c:
            c.upload(p, u)
            c.step(50)
            wp, wu = c.download()
            ws = c.stats()
        assert np.array_equal(gp, wp) and np.array_equal(gu, wu)
        np.testing.assert_allclose(s["solute"], ws["solute"], rtol=1e-12)


def test_autotune_restores_state_and_caches(tmp_path):
    m, phi, mu = mb.load_case(BINARY["iso"])
    cache = str(tmp_path / "tiles.txt")
    with mb.Batch([m]) as b:
        b.upload(0, phi, mu)
        b.step(3)
        before = b.download(0)
        tx, ty = b.autotune(cache)
        after = b.download(0)
        assert (tx, ty) in [(16, 32), (8, 32), (32, 32), (16, 64)]
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
        assert os.path.exists(cache) and len(open(cache).read().split()) == 14
        assert b.autotune(cache) == (tx, ty)  # read back from the cache


def test_tip_velocity_within_half_percent_of_fp64():
    """The accuracy bar of the FP32 form on a reduced corner dendrite (256^2, 8,000 steps): the
    FP32 form's tip velocity within 0.5% of the FP64 form's, solute mass within
    1e-4 (the full 1024^2 x 50,000-step run: python -m microsim_b200.validate)."""
    from microsim_b200 import validate
    r = validate.compare(mesh=256, steps=8000, every=500)
    assert r["nonfinite"] == 0
    assert r["tip_velocity_fp64"] > 0
    assert r["tip_velocity_rel_err"] <= 5e-3
    assert r["tip_position_rel_err"] <= 1e-3
    assert r["solute_rel_diff"] <= 1e-4


def test_batched_sweep_subset_within_half_percent_of_fp64():
    """A 32-instance sub-sweep of the batched-sweep workload (sides 128..512, uneven
    parameters), 1,000 steps: every instance's FP32 tip velocity within 0.5% of the FP64
    plain form's, solute mass within 1e-4 (the full 256 x 5,000-step run:
    python -m microsim_b200.validate --workload c4)."""
    from microsim_b200 import validate
    r = validate.compare("c4", steps=1000, every=100, instances=32)
    assert r["instances"] == 32
    assert r["nonfinite_max"] == 0
    assert r["tip_velocity_rel_err_max"] <= 5e-3, r
    assert r["solute_rel_diff_max"] <= 1e-4, r


def test_narrow_band_is_bit_identical_to_the_full_kernel():
    """Tiles sent to the lean pure-phase kernel get the same bits as from the
    full kernel, for every tile shape: Neumann borders (mirrored rings), a
    periodic batch member (wrapped rings are never trusted), a periodic mu under
    Neumann phi (ghosts of lean edge tiles from the far side), partial edge tiles
    with fewer than three cells on an axis, the skipped phi writes, and a
    re-upload in mid-run (purity words reset)."""
    cases = [configs.binary_case(200, 150, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(0, 0, 8.0)),
             configs.binary_case(160, 224, gap=1.0, supersat=0.4, eps=3.0, delta=0.03, theta=15.0, dt=0.05,
                                 tau=1.3332, seed=(80, 100, 9.0), bc=(3, 3, 3, 3)),
             configs.binary_case(98, 130, gap=1.0, supersat=0.5, eps=4.0, delta=0.01, dt=0.05, tau=1.7776,
                                 seed=(49, 65, 7.0))]
    loaded = [mb.load_case(c) for c in cases]
    # Neumann phi with a periodic mu: the lean tiles' ghost rows/columns come from the far side
    m4, p4, u4 = mb.load_case(cases[0])
    m4 = m4.copy()
    for i in range(4):
        m4.bc_mu[i] = 3
    loaded.append((m4, p4, u4))
    models = [m for m, _, _ in loaded]

    def run(on, tile, reupload=False, scan=False):
        with mb.Batch(models) as b:
            b.set_tile(*tile)
            b.set_narrowband(on)
            b.set_scan(scan)
            for i, (_, p, u) in enumerate(loaded):
                b.upload(i, p, u)
            b.step(150)  # graph replays and direct launches, both buffer parities
            if reupload:
                for i, st in enumerate([b.download(i) for i in range(len(models))]):
                    b.upload(i, *st)
            b.step(151)
            lean = b.lean_tiles()
            return [b.download(i) for i in range(len(models))], lean

    ref, (lean0, _) = run(False, (16, 32))
    assert lean0 == 0
    for tile, scan in [((16, 32), False), ((8, 32), False), ((32, 32), False), ((16, 64), False),
                       ((16, 32), True), ((8, 32), True)]:
        got, (lean, total) = run(True, tile, reupload=tile == (16, 32), scan=scan)
        assert lean > total // 2, (tile, lean, total)  # the lean kernel does most of the work
        for (p1, u1), (p0, u0) in zip(got, ref):
            assert np.array_equal(p1, p0) and np.array_equal(u1, u0), tile
    # four phases, two chemical potentials: pure grains of every solid phase and the liquid
    m, phi, mu = mb.load_case(configs.c3(steps=200, mesh=160, nseeds=6, rng_seed=7))
    res = []
    for on in (True, False):
        with mb.Batch([m]) as b:
            b.set_narrowband(on)
            b.upload(0, phi, mu)
            b.step(120)
            res.append((b.download(0), b.lean_tiles()))
    (a, la), (c, lc) = res
    assert la[0] > 0 and lc[0] == 0
    assert np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1])


def test_two_step_blocking_is_bit_identical_to_single_steps():
    """Blocked pairs (the lean tiles two diffusion steps per staged box, the other
    tiles through the full kernel twice via the intermediate buffer) give the bits of
    single steps, for every tile shape: Neumann borders (two-deep mirrored boxes and
    the intermediate step's ghosts), a periodic member (its border tiles take the full
    kernel), a periodic mu under Neumann phi, partial edge tiles (1- and 2-cell
    remainders), odd step counts (a single step after the pairs), graph replays of
    both parities, re-uploads, and a four-phase ternary case."""
    cases = [configs.binary_case(200, 150, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(0, 0, 8.0)),
             configs.binary_case(160, 224, gap=1.0, supersat=0.4, eps=3.0, delta=0.03, theta=15.0, dt=0.05,
                                 tau=1.3332, seed=(80, 100, 9.0), bc=(3, 3, 3, 3)),
             configs.binary_case(98, 130, gap=1.0, supersat=0.5, eps=4.0, delta=0.01, dt=0.05, tau=1.7776,
                                 seed=(49, 65, 7.0)),
             configs.binary_case(129, 161, gap=1.0, supersat=0.5, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(128, 160, 10.0)),
             configs.binary_case(145, 98, gap=1.0, supersat=0.45, eps=3.0, delta=0.015, dt=0.05, tau=1.3332,
                                 seed=(70, 0, 9.0))]
    loaded = [mb.load_case(c) for c in cases]
    m4, p4, u4 = mb.load_case(cases[0])
    m4 = m4.copy()
    for i in range(4):
        m4.bc_mu[i] = 3
    loaded.append((m4, p4, u4))
    models = [m for m, _, _ in loaded]

    def run(depth, tile, reupload=False):
        with mb.Batch(models) as b:
            b.set_tile(*tile)
            b.set_depth(depth)
            assert b.depth() == depth
            for i, (_, p, u) in enumerate(loaded):
                b.upload(i, p, u)
            b.step(150)  # 4-step graphs of both parities, then pairs
            if reupload:
                for i, st in enumerate([b.download(i) for i in range(len(models))]):
                    b.upload(i, *st)
            b.step(151)  # odd: pairs and one single step
            lean = b.lean_tiles()
            return [b.download(i) for i in range(len(models))], lean

    for tile in [(16, 32), (8, 32), (32, 32), (16, 64)]:
        ref, _ = run(1, tile)
        got, (lean, total) = run(2, tile, reupload=tile == (16, 32))
        assert lean > total // 2, (tile, lean, total)
        for i, ((p1, u1), (p0, u0)) in enumerate(zip(got, ref)):
            assert np.array_equal(p1, p0) and np.array_equal(u1, u0), (tile, i, np.abs(u1 - u0).max())
    m, phi, mu = mb.load_case(configs.c3(steps=200, mesh=160, nseeds=6, rng_seed=7))
    res = []
    for depth in (2, 1):
        with mb.Batch([m]) as b:
            b.set_depth(depth)
            b.upload(0, phi, mu)
            b.step(120)
            res.append(b.download(0))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def _golden_model(name):
    g = load_golden(name)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    return g, m, phi, mu


def test_nonisothermal_batch_equals_contexts_and_resumes():
    """The frozen temperature gradient in the FP32 batch: two instances with their own gradients
    (one moving), single steps and blocked pairs, equal FP32 contexts bit for bit; the
    statistics see each instance's temperature; a batch resumed at step 20 with
    set_time_step(20) continues the run bit for bit; and it stays within the FP32 tolerance
    of the FP64 form."""
    g, m, phi, mu = _golden_model("tempgrad_aniso_bin")
    m2 = m.copy()
    m2.tg_velocity = 0.0  # a second instance with a frozen (not moving) gradient
    m2.tg_offset = m.tg_offset + 3.0
    models, steps = [m, m2], 41
    ref = []
    for mm in models:
        with mb.Context(mm, mb.GP_FP32) as c:
            c.upload(phi, mu)
            c.step(steps)
            ref.append((*c.download(), c.stats()))
    for depth in (1, 2):
        with mb.Batch(models) as b:
            b.set_depth(depth)
            for i in range(2):
                b.upload(i, phi, mu)
            b.step(steps)
            for i in range(2):
                p, u = b.download(i)
                assert np.array_equal(p, ref[i][0]) and np.array_equal(u, ref[i][1]), (depth, i)
                np.testing.assert_allclose(b.stats(i)["solute"], ref[i][2]["solute"], rtol=1e-12)
    assert not np.array_equal(ref[0][1], ref[1][1])  # the two gradients differ
    with mb.Batch(models) as b:
        for i in range(2):
            b.upload(i, phi, mu)
        b.step(20)
        mid = [b.download(i) for i in range(2)]
    with mb.Batch(models) as b:
        for i in range(2):
            b.upload(i, *mid[i])
        b.set_time_step(20)
        b.step(steps - 20)
        for i in range(2):
            p, u = b.download(i)
            assert np.array_equal(p, ref[i][0]) and np.array_equal(u, ref[i][1]), i
    with mb.Context(m, mb.GP_FP64) as c64:
        c64.upload(phi, mu)
        c64.step(steps)
        p64, u64 = c64.download()
    assert np.abs(ref[0][0] - p64).max() <= 1e-4
    assert np.abs(ref[0][1] - u64).max() <= 1e-3
    # compensated accumulation under the gradient, blocked pairs: still within the tolerance
    with mb.Batch(models) as b:
        b.set_compensated(True)
        b.set_depth(2)
        for i in range(2):
            b.upload(i, phi, mu)
        b.step(steps)
        pc, uc = b.download(0)
    assert np.abs(pc - p64).max() <= 1e-4 and np.abs(uc - u64).max() <= 1e-3


def test_isotropic_and_anisotropic_instances_in_one_batch():
    """A batch mixing isotropic and anisotropic instances runs the anisotropic kernels with no
    anisotropy for the isotropic ones: the anisotropic instances equal their own FP32 contexts bit
    for bit; the isotropic ones go through the anisotropic kernel's (mathematically equal)
    arithmetic and agree with their isotropic contexts to FP32 rounding."""
    cases = [configs.binary_case(64, 48, gap=1.0, supersat=0.5, eps=4.0, dt=0.05, tau=1.7776, seed=(32, 24, 8.0)),
             BINARY["aniso_corner"],
             configs.binary_case(48, 80, gap=1.0, supersat=0.45, eps=3.0, dt=0.05, tau=1.3332, seed=(24, 40, 7.0),
                                 bc=(3, 3, 3, 3))]
    loaded = [mb.load_case(c) for c in cases]
    assert [int(m.anisotropy) for m, _, _ in loaded] == [0, 1, 0]
    ref = []
    for m, phi, mu in loaded:
        with mb.Context(m, mb.GP_FP32) as c:
            c.upload(phi, mu)
            c.step(200)
            ref.append(c.download())
    for depth in (1, 2):
        with mb.Batch([m for m, _, _ in loaded]) as b:
            b.set_depth(depth)
            for i, (_, phi, mu) in enumerate(loaded):
                b.upload(i, phi, mu)
            b.step(200)
            for i, (p0, u0) in enumerate(ref):
                p1, u1 = b.download(i)
                if loaded[i][0].anisotropy:
                    assert np.array_equal(p1, p0) and np.array_equal(u1, u0), (depth, i)
                else:
                    assert np.abs(p1 - p0).max() <= 1e-5 and np.abs(u1 - u0).max() <= 1e-5, (depth, i)


def test_queued_statistics_equal_the_waiting_ones():
    """Statistics read back queued after every step (no host wait per step, one sync at the end)
    decode to exactly what the waiting call returns after the same steps, for every instance."""
    cases = [configs.binary_case(96, 64, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(0, 0, 8.0)),
             configs.binary_case(160, 128, gap=1.0, supersat=0.5, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(80, 64, 9.0))]
    loaded = [mb.load_case(c) for c in cases]
    models = [m for m, _, _ in loaded]
    import torch
    steps = 12
    raw = torch.zeros((steps, len(models), mb.GP_STAT_VALUES), dtype=torch.float64, pin_memory=True).numpy()
    want = []
    with mb.Batch(models) as b:
        for i, (_, p, u) in enumerate(loaded):
            b.upload(i, p, u)
        for t in range(steps):
            b.step(1)
            want.append([b.stats(i) for i in range(len(models))])
    with mb.Batch(models) as b:
        for i, (_, p, u) in enumerate(loaded):
            b.upload(i, p, u)
        for t in range(steps):
            b.step(1)
            for i in range(len(models)):
                b.stats_async(i, raw[t, i])
        b.sync()
        for t in range(steps):
            for i in range(len(models)):
                got = b.stats_from_raw(i, raw[t, i])
                for k, v in want[t][i].items():
                    assert np.array_equal(np.asarray(got[k]), np.asarray(v)), (t, i, k)
        with pytest.raises(ValueError):
            b.stats_async(0, np.zeros(8))


def test_async_upload_download_equal_the_waiting_ones():
    """Queued uploads and downloads of every instance (no host wait between instances, one sync),
    through the staging buffer (pageable arrays) or read and written in place by the conversion
    kernels (page-locked arrays), give the state the waiting calls give."""
    cases = [configs.binary_case(96, 64, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(0, 0, 8.0)),
             configs.binary_case(160, 128, gap=1.0, supersat=0.5, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(80, 64, 9.0))]
    loaded = [mb.load_case(c) for c in cases]
    models = [m for m, _, _ in loaded]
    import torch

    def pinned(a):  # page-locked host array: the queued copies read / write it in place
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    res = []
    for wait, pin in ((True, False), (False, False), (False, True)):
        held = [((pinned(p), pinned(u)) if pin else (np.ascontiguousarray(p), np.ascontiguousarray(u)))
                for _, p, u in loaded]  # alive until sync
        with mb.Batch(models) as b:
            for i, (p, u) in enumerate(held):
                b.upload(i, p, u, wait=wait)
            b.step(30)
            outs = [b.download(i, *((pinned(np.zeros_like(p)), pinned(np.zeros_like(u))) if pin else (None, None)),
                               wait=wait) for i, (p, u) in enumerate(held)]
            b.sync()
            res.append([(p.copy(), u.copy()) for p, u in outs])
    # every instance at once: one page-locked instance and one pageable, mixed
    held = [(pinned(loaded[0][1]), pinned(loaded[0][2])),
            (np.ascontiguousarray(loaded[1][1]), np.ascontiguousarray(loaded[1][2]))]
    outs = [(pinned(np.zeros_like(held[0][0])), pinned(np.zeros_like(held[0][1]))),
            (np.zeros_like(held[1][0]), np.zeros_like(held[1][1]))]
    with mb.Batch(models) as b:
        b.upload_all(held)
        b.step(30)
        b.download_all(outs)
        b.sync()
        res.append([(p.copy(), u.copy()) for p, u in outs])
    for r in res[1:]:
        for (p1, u1), (p0, u0) in zip(r, res[0]):
            assert np.array_equal(p1, p0) and np.array_equal(u1, u0)


def test_compensated_accumulation():
    """Compensated (TwoSum/TwoProduct) accumulation: on for a context and a batch,
    refused for FP64; the results change bits, stay within the FP32 tolerances of
    the FP64 form, and stay bit-identical across the narrow band, tile shapes and
    two-step blocking (every kernel shares the compensated pure-phase rule)."""
    m, phi, mu = mb.load_case(BINARY["aniso_corner"])
    with mb.Context(m, mb.GP_FP64) as c64:
        with pytest.raises(RuntimeError):
            c64.set_compensated(True)
        assert not c64.compensated()
        c64.upload(phi, mu)
        c64.step(400)
        p64, u64 = c64.download()
        s64 = c64.stats()
    res = {}
    for comp in (False, True):
        with mb.Context(m, mb.GP_FP32) as c:
            c.set_compensated(comp)
            assert c.compensated() == comp
            c.upload(phi, mu)
            c.step(400)
            res[comp] = (*c.download(), c.stats())
    assert not np.array_equal(res[True][1], res[False][1])
    p32, u32, s32 = res[True]
    assert np.abs(p32 - p64).max() <= 2e-5
    assert np.abs(u32 - u64).max() <= 1e-4
    np.testing.assert_allclose(s32["solute"], s64["solute"], rtol=1e-4)

    cases = [configs.binary_case(200, 150, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(0, 0, 8.0)),
             configs.binary_case(129, 161, gap=1.0, supersat=0.5, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                                 seed=(128, 160, 10.0))]
    loaded = [mb.load_case(c) for c in cases]
    models = [mm for mm, _, _ in loaded]

    def run(nb, depth, tile):
        with mb.Batch(models) as b:
            b.set_compensated(True)
            assert b.compensated()
            b.set_tile(*tile)
            b.set_narrowband(nb)
            b.set_depth(depth)
            for i, (_, p, u) in enumerate(loaded):
                b.upload(i, p, u)
            b.step(101)
            return [b.download(i) for i in range(len(models))]

    ref = run(False, 1, (16, 32))
    for nb, depth, tile in [(True, 1, (16, 32)), (True, 2, (16, 32)), (True, 2, (8, 32)), (True, 1, (32, 32))]:
        for (p1, u1), (p0, u0) in zip(run(nb, depth, tile), ref):
            assert np.array_equal(p1, p0) and np.array_equal(u1, u0), (nb, depth, tile)


def test_two_step_blocking_timing_and_stats():
    """Per-kernel timing of blocked pairs covers two steps per launch set, and the
    statistics read after pairs see the blocked state."""
    m, phi, mu = mb.load_case(configs.binary_case(256, 256, gap=1.0, supersat=0.5, eps=4.0, delta=0.02, dt=0.05,
                                                  tau=1.7776, seed=(0, 0, 12.0)))
    with mb.Batch([m, m]) as b:
        b.set_depth(2)
        for i in range(2):
            b.upload(i, phi, mu)
        b.set_timing(True)
        b.step(10)
        kt = b.kernel_ms()
        b.set_timing(False)
        assert kt["steps"] == 10 and kt["lean"] > 0 and kt["general"] > 0
        st = b.stats(0)
        assert st["nonfinite"] == 0 and st["rel_change_mu"][0] > 0


def test_grid_split_and_prepared_graphs_are_bit_identical():
    """The persistent grids' blocks per SM (lean and full kernels, run
    concurrently), the full kernel's block size, the scan or list way of finding
    the interface tiles and graph capture ahead of time change no bits; prepare()
    takes no step."""
    m, phi, mu = mb.load_case(BINARY["aniso_corner"])
    res = []
    for grids, prep, block, scan in [((0, 0), False, 256, False), ((1, 1), True, 512, True),
                                     ((2, 3), True, 256, True), ((0, 2), False, 512, False)]:
        with mb.Batch([m, m]) as b:
            b.set_block(block)
            b.set_scan(scan)
            assert b.block() == block and b.scan() == scan
            b.set_grids(*grids)
            lp, gp, occ_l, occ_g = b.grids()
            assert lp == (grids[0] if 0 < grids[0] < occ_l else occ_l)
            assert gp == (grids[1] if 0 < grids[1] < occ_g else occ_g)
            b.upload(0, phi, mu)
            b.upload(1, phi, mu)
            if prep:
                before = b.download(0)
                b.prepare()
                after = b.download(0)
                assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
            b.step(37)
            res.append(b.download(1))
    for p, u in res[1:]:
        assert np.array_equal(p, res[0][0]) and np.array_equal(u, res[0][1])


def test_moving_frame_within_tolerance_of_reference():
    """Shift = 1 in the FP32 form: same interface rows and offsets as the
    reference, fields within the 2-phase tolerances (the first step after a
    shift reads ghost rows through the boundary map)."""
    g = load_golden("shift_planar")
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
    offset, done, k = 0, 0, 0
    with mb.Context(m, mb.GP_FP32) as c:
        c.upload(phi, mu)
        for t in g["dump_steps"]:
            t = int(t)
            while done < t:
                nxt = min(t, (done // 100 + 1) * 100)
                c.step(nxt - done)
                done = nxt
                if done % 100 == 0:
                    pos = c.interface_y()
                    assert pos == g["shifts"][k][1]
                    if pos > 20:
                        c.shift_y(pos - 20)
                        offset += pos - 20
                    assert offset == g["shifts"][k][2]
                    k += 1
            p, u = c.download()
            assert np.abs(p - interior(g[f"phi_{t}"])).max() <= 1e-4, t
            assert np.abs(u - interior(g[f"mu_{t}"])).max() <= 1e-3, t
