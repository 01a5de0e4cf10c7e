"""Energies of a state: gp_stats' FP64 energy sums and their numpy checker.

The reference prints no global energy; gp_stats integrates the functional whose
phi-derivatives its phase-field step uses (gradient energy, obstacle/well
potential, chemical free energy and grand potential; the definitions sit in
include/gp_b200.h beside gp_stats).  The CPU tests pin the numpy checker
(oracle.gp_oracle.energies) on states whose energies follow by hand from the
reference's formulas; the GPU tests compare the device sums, FP64 and FP32
contexts, with the checker on the reference's own states (golden fixtures).
"""
import tempfile

import numpy as np
import pytest

from conftest import isothermal_cases, interior, load_golden, write_inputs
import microsim_b200 as mb
from oracle import gp_oracle as O


def _c(N=2, K1=1, obstacle=1, aniso=0, bc=(1, 1), eps=4.0, dx=1.0, dy=1.0):
    c = {"N": N, "K1": K1, "dx": dx, "dy": dy, "epsilon": eps, "obstacle": obstacle, "anisotropy": aniso,
         "bc_phi": bc, "Gamma": np.ones((N, N)), "Gamma_abc": np.zeros((N, N, N)), "dab": np.zeros((N, N)),
         "R": np.tile(np.eye(2), (N, N, 1, 1)), "cmu": np.ones((N, K1, K1)) * 0.5, "A": np.ones((N, K1, K1)),
         "Beff": np.zeros((N, K1)), "B": np.zeros((N, K1)), "C": np.zeros(N)}
    return c


def test_gradient_energy_of_a_linear_ramp():
    # phi_0 rises linearly along x (slope s), phi_1 = 1 - phi_0: q_01 = -grad phi_0, |q|^2 = s^2;
    # Neumann mirrors make the centred gradient of the first/last row zero.
    mx, my, s = 12, 5, 0.05
    p0 = np.repeat((0.2 + s * np.arange(mx))[:, None], my, axis=1)
    phi = np.stack([p0, 1 - p0])
    mu = np.zeros((1, mx, my))
    c = _c(eps=3.0)
    e = O.energies(c, phi, mu)
    assert np.isclose(e["energy_gradient"], 3.0 * s * s * (mx - 2) * my, rtol=1e-12)


def test_potentials_of_a_uniform_mixture():
    mx, my = 6, 7
    phi = np.full((2, mx, my), 0.5)
    mu = np.zeros((1, mx, my))
    for obstacle, w in ((1, 16.0 / np.pi ** 2 * 0.25), (0, 9.0 * 0.0625)):
        e = O.energies(_c(obstacle=obstacle, eps=2.0), phi, mu)
        assert np.isclose(e["energy_potential"], w / 2.0 * mx * my, rtol=1e-14)
        assert e["energy_gradient"] == 0.0
    # a triple junction term: three phases at 1/3 with Gamma_abc = 2
    phi3 = np.full((3, mx, my), 1.0 / 3.0)
    c3 = _c(N=3, obstacle=1, eps=1.0)
    c3["Gamma_abc"][0][1][2] = 2.0
    e = O.energies(c3, phi3, np.zeros((1, mx, my)))
    want = (16.0 / np.pi ** 2 * 3 * (1 / 9) + 2.0 / 27) * mx * my
    assert np.isclose(e["energy_potential"], want, rtol=1e-13)


def test_chemical_energy_of_pure_phases():
    # pure phase a: h_a = 1, c = cmu (mu - Beff), f = A c^2 + B c + C (functionF_01.h:5-18)
    mx, my = 4, 4
    c = _c()
    c["A"][1][0][0], c["B"][1][0], c["C"][1], c["Beff"][1][0], c["cmu"][1][0][0] = 2.0, 0.3, -0.1, 0.2, 0.25
    phi = np.zeros((2, mx, my))
    phi[1] = 1.0
    mu = np.full((1, mx, my), 0.6)
    conc = 0.25 * (0.6 - 0.2)
    f = 2.0 * conc * conc + 0.3 * conc - 0.1
    e = O.energies(c, phi, mu)
    assert np.isclose(e["energy_chemical"], f * mx * my, rtol=1e-14)
    assert np.isclose(e["grand_potential"], (f - 0.6 * conc) * mx * my, rtol=1e-14)
    assert e["energy_potential"] == 0.0 and e["energy_gradient"] == 0.0


def _model_dict(m):
    N, K1 = m.N, m.K1
    return {"N": N, "K1": K1, "dx": m.dx, "dy": m.dy, "epsilon": m.epsilon, "obstacle": m.obstacle,
            "anisotropy": m.anisotropy, "bc_phi": (m.bc_phi[0], m.bc_phi[3]),
            "Gamma": m.arr("Gamma")[:N, :N], "Gamma_abc": m.arr("Gamma_abc")[:N, :N, :N],
            "dab": m.arr("dab")[:N, :N], "R": m.arr("R")[:N, :N], "cmu": m.arr("cmu")[:N, :K1, :K1],
            "A": m.arr("A")[:N, :K1, :K1], "Beff": m.arr("Beff")[:N, :K1], "B": m.arr("B")[:N, :K1],
            "C": m.arr("C")[:N]}


def _case_state(case):
    g = load_golden(case)
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        m = mb.Input(ip, fp).model()
    last = int(g["dump_steps"][-1])
    return m, interior(g["phi_%d" % last]).copy(), interior(g["mu_%d" % last]).copy()


def _check(got, want, ncell):
    for k in ("energy_gradient", "energy_potential", "energy_chemical", "grand_potential"):
        assert abs(got[k] - want[k]) <= 1e-11 * ncell + 1e-11 * abs(want[k]), (k, got[k], want[k])


@pytest.mark.gpu
@pytest.mark.parametrize("case", isothermal_cases())
def test_device_energies_match_the_checker_fp64(case):
    m, phi, mu = _case_state(case)
    with mb.Context(m, mb.GP_FP64) as ctx:
        ctx.upload(phi, mu)
        got = ctx.stats()
    _check(got, O.energies(_model_dict(m), phi, mu), phi.shape[1] * phi.shape[2])
    assert got["free_energy"] == got["energy_gradient"] + got["energy_potential"] + got["energy_chemical"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", isothermal_cases())
def test_device_energies_match_the_checker_fp32_batch(case):
    m, phi, mu = _case_state(case)
    try:
        b = mb.Batch([m])
    except mb.GpError as e:
        if e.rc == mb.GP_E_UNSUPPORTED:
            pytest.skip("no FP32 kernels for this N, K1")
        raise
    with b:
        b.upload(0, phi, mu)
        got = b.stats(0)
    # the batch stores FP32 and sums in FP64: the checker on the FP32-rounded fields
    f32 = lambda a: a.astype(np.float32).astype(np.float64)
    _check(got, O.energies(_model_dict(m), f32(phi), f32(mu)), phi.shape[1] * phi.shape[2])
