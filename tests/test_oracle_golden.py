"""The oracle restatement against the reference itself (tests/golden fixtures).

Bit-exact: every fixture was produced by the reference serial solver compiled
from its own sources; the C restatement must reproduce its doubles exactly on
the interior and on the Delta-phi ring the interior reads.
"""
import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, oracle_model
from oracle import gp_oracle as O


def start_state(g, m):
    """The fixture's state before its first time step: the filled domain, after
    the NSMOOTH - 1 smoothing pre-steps when the input asks for them."""
    phi, mu = g["phi_0"].copy(), g["mu_0"].copy()
    if "nsmooth" in g:
        O.smooth(m, phi, mu, int(g["nsmooth"]) - 1)
    return phi, mu


@pytest.mark.parametrize("case", [c for c in golden_cases() if "nsmooth" in load_golden(c)])
def test_smoothing_pre_steps_bitexact(case):
    g = load_golden(case)
    phi, mu = start_state(g, oracle_model(g))
    assert np.array_equal(interior(phi), interior(g["phi_smoothed"]))
    assert np.array_equal(interior(mu), interior(g["mu_smoothed"]))
    assert np.array_equal(phi, g["phi_smoothed"]) and np.array_equal(mu, g["mu_smoothed"])  # ghosts too


@pytest.mark.parametrize("case", golden_cases())
def test_dphi_first_step_bitexact(case):
    g = load_golden(case)
    m = oracle_model(g)
    phi, mu = start_state(g, m)
    dphi, _ = O.step(m, phi, mu, 1, want_dphi=True)
    ring = (slice(None), slice(2, -2), slice(2, -2))
    assert np.array_equal(dphi[ring], g["dphi_1"][ring]), \
        f"max |diff| {np.abs(dphi[ring] - g['dphi_1'][ring]).max()}"


@pytest.mark.parametrize("case", golden_cases())
def test_states_bitexact(case):
    g = load_golden(case)
    m = oracle_model(g)
    phi, mu = start_state(g, m)
    done = 0
    for t in g["dump_steps"]:
        O.step(m, phi, mu, int(t) - done)
        done = int(t)
        assert np.array_equal(interior(phi), interior(g[f"phi_{t}"])), f"phi differs after step {t}"
        assert np.array_equal(interior(mu), interior(g[f"mu_{t}"])), f"mu differs after step {t}"


@pytest.mark.parametrize("case", golden_cases())
def test_ghost_fill_matches(case):
    """Ghost layers after the boundary copy equal the reference's (t = 0 and later)."""
    g = load_golden(case)
    m = oracle_model(g)
    phi, mu = g["phi_0"].copy(), g["mu_0"].copy()
    phi[:, :3, :] = 0; phi[:, -3:, :] = 0; phi[:, :, :3] = 0; phi[:, :, -3:] = 0
    mu[:, :3, :] = 0; mu[:, -3:, :] = 0; mu[:, :, :3] = 0; mu[:, :, -3:] = 0
    O.apply_bc(m, phi, mu)
    assert np.array_equal(phi, g["phi_0"]) and np.array_equal(mu, g["mu_0"])


def test_oracle_rejects_unsupported_boundary():
    g = load_golden("iso_obst_bin")
    m = oracle_model(g)
    m.bc_phi = (0, 0, 1, 1)
    with pytest.raises(ValueError):
        O.step(m, g["phi_0"].copy(), g["mu_0"].copy(), 1)
