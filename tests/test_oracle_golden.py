"""The oracle restatement against the reference itself (tests/golden fixtures).

Bit-exact: every fixture was produced by the reference serial solver compiled
from its own sources; the C restatement must reproduce its doubles exactly on
the interior and on the Delta-phi ring the interior reads.
"""
import numpy as np
import pytest

from conftest import isothermal_cases, interior, load_golden, oracle_model
from oracle import gp_oracle as O


def start_state(g, m):
    """The fixture's state before its first time step: the filled domain, after
    the NSMOOTH - 1 smoothing pre-steps when the input asks for them."""
    phi, mu = g["phi_0"].copy(), g["mu_0"].copy()
    if "nsmooth" in g:
        O.smooth(m, phi, mu, int(g["nsmooth"]) - 1)
    return phi, mu


@pytest.mark.parametrize("case", [c for c in isothermal_cases() if "nsmooth" in load_golden(c)])
def test_smoothing_pre_steps_bitexact(case):
    g = load_golden(case)
    phi, mu = start_state(g, oracle_model(g))
    assert np.array_equal(interior(phi), interior(g["phi_smoothed"]))
    assert np.array_equal(interior(mu), interior(g["mu_smoothed"]))
    assert np.array_equal(phi, g["phi_smoothed"]) and np.array_equal(mu, g["mu_smoothed"])  # ghosts too


@pytest.mark.parametrize("case", isothermal_cases())
def test_dphi_first_step_bitexact(case):
    g = load_golden(case)
    m = oracle_model(g)
    phi, mu = start_state(g, m)
    dphi, _ = O.step(m, phi, mu, 1, want_dphi=True)
    ring = (slice(None), slice(2, -2), slice(2, -2))
    assert np.array_equal(dphi[ring], g["dphi_1"][ring]), \
        f"max |diff| {np.abs(dphi[ring] - g['dphi_1'][ring]).max()}"


def interface_row(m, phi):
    """check_SHIFT (functions/shift.h:43-66) over the interior columns of the
    ghost-padded fields: the highest row y where the liquid fraction crosses 0.5
    between rows y-1 and y."""
    pl = phi[m.N - 1, 3:-3, :]
    f = pl - (1.0 - pl)
    hit = (f[:, :-1] < 0.0) & (f[:, 1:] > 0.0)
    ys = np.nonzero(hit.any(axis=0))[0]
    return int(ys.max() + 1) if ys.size else 0


def shift_rows(m, phi, mu, d, mu_fill):
    """apply_shiftY (functions/shift.h:4-40) on the ghost-padded fields, ghost
    rows included, no boundary copy afterwards (as the reference's main)."""
    ry = phi.shape[2]
    phi[:, :, : ry - d] = phi[:, :, d:].copy()
    mu[:, :, : ry - d] = mu[:, :, d:].copy()
    phi[:, :, ry - d:] = 0.0
    phi[m.N - 1, :, ry - d:] = 1.0
    mu[:, :, ry - d:] = np.asarray(mu_fill)[:, None, None]


def liquid_fill_mu(g):
    import tempfile
    import microsim_b200 as mb
    from conftest import write_inputs
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        mdl = mb.Input(ip, fp).model()
    return np.array(mdl.mu_shift[: mdl.K1])


@pytest.mark.parametrize("case", isothermal_cases())
def test_states_bitexact(case):
    """Including the moving frame: the interface row of every 100th step equals
    the reference's, and shifting the ghost-padded fields as the reference does
    keeps the states bit-exact."""
    g = load_golden(case)
    m = oracle_model(g)
    phi, mu = start_state(g, m)
    shifts = g.get("shifts")
    mu_fill = liquid_fill_mu(g) if shifts is not None else None
    shiftj = int(str(g["input_text"]).split("Shiftj = ")[1].split(";")[0]) if shifts is not None else 0
    done, k = 0, 0
    for t in g["dump_steps"]:
        while done < int(t):
            nxt = min(int(t), (done // 100 + 1) * 100) if shifts is not None else int(t)
            O.step(m, phi, mu, nxt - done)
            done = nxt
            if shifts is not None and done % 100 == 0:
                pos = interface_row(m, phi)
                assert pos == shifts[k][1], (done, pos, shifts[k])
                if pos > shiftj:
                    shift_rows(m, phi, mu, pos - shiftj, mu_fill)
                k += 1
        assert np.array_equal(interior(phi), interior(g[f"phi_{t}"])), f"phi differs after step {t}"
        assert np.array_equal(interior(mu), interior(g[f"mu_{t}"])), f"mu differs after step {t}"


@pytest.mark.parametrize("case", isothermal_cases())
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
