"""Host side of the drop-in (C library, no GPU): Input.in parsing, model
constants, filling and VTK bytes, against the reference's own outputs."""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, write_inputs
import microsim_b200 as mb


def _parse(g, d):
    ip, fp = write_inputs(g, d)
    inp = mb.Input(ip, fp)
    return inp, inp.model()


@pytest.mark.parametrize("case", golden_cases())
def test_model_constants_bitexact(case):
    g = load_golden(case)
    with tempfile.TemporaryDirectory() as d:
        inp, m = _parse(g, d)
    N, K1 = m.N, m.K1
    assert N == int(g["c_NUMPHASES"][0]) and K1 == int(g["c_NUMCOMPONENTS"][0]) - 1
    eq = np.array_equal
    assert eq(m.arr("cmu")[:N, :K1, :K1], g["c_cmu"].reshape(N, K1, K1))
    assert eq(m.arr("A")[:N, :K1, :K1], g["c_A"].reshape(N, K1, K1))
    assert eq(m.arr("Diff")[:N, :K1, :K1], g["c_Diffusivity"].reshape(N, K1, K1))
    assert eq(m.arr("B")[:N, :K1], g["c_B"].reshape(N, K1))
    assert eq(m.arr("C")[:N], g["c_C"])
    beff = g["c_Beq"].reshape(N, K1) + g["c_dBbdT"].reshape(N, K1) * (g["c_T"][0] - g["c_Teq"][0])
    assert eq(m.arr("Beff")[:N, :K1], beff)
    assert eq(m.arr("Gamma")[:N, :N], g["c_Gamma"].reshape(N, N))
    assert eq(m.arr("tau_ab")[:N, :N], g["c_tau_ab"].reshape(N, N))
    assert m.obstacle == int(g["c_OBSTACLE"][0]) and m.anisotropy == int(g["c_ANISOTROPY"][0])
    if m.anisotropy:
        assert eq(m.arr("dab")[:N, :N], g["c_dab"].reshape(N, N))
        R = g["c_Rotation_matrix"].reshape(N, N, 3, 3)[:, :, :2, :2]
        Ri = g["c_Inv_Rotation_matrix"].reshape(N, N, 3, 3)[:, :, :2, :2]
        assert eq(m.arr("R")[:N, :N], R)
        assert eq(m.arr("Rinv")[:N, :N], Ri)
    if N >= 3:
        assert eq(m.arr("Gamma_abc")[:N, :N, :N], g["c_Gamma_abc"].reshape(N, N, N))
    assert tuple(m.bc_phi) == tuple(int(v) for v in g["c_bc_phi"])
    assert tuple(m.bc_mu) == tuple(int(v) for v in g["c_bc_mu"])
    assert (m.dx, m.dy, m.dt, m.epsilon, m.tau) == (g["c_deltax"][0], g["c_deltay"][0], g["c_deltat"][0],
                                                    g["c_epsilon"][0], g["c_tau"][0])


@pytest.mark.parametrize("case", golden_cases())
def test_fill_bitexact(case):
    g = load_golden(case)
    with tempfile.TemporaryDirectory() as d:
        inp, m = _parse(g, d)
        phi, mu = inp.fill(m)
    assert np.array_equal(phi, interior(g["phi_0"]))
    assert np.array_equal(mu, interior(g["mu_0"]))


@pytest.mark.parametrize("case", golden_cases())
def test_vtk_bytes_identical(case):
    g = load_golden(case)
    with tempfile.TemporaryDirectory() as d:
        inp, m = _parse(g, d)
        path = os.path.join(d, "out_0.vtk")
        inp.write_vtk(m, path, interior(g["phi_0"]), interior(g["mu_0"]))
        data = open(path, "rb").read()
        assert data == g["vtk_0"].tobytes()
        phi, mu = inp.read_vtk(m, path)
    if str(g["input_text"]).find("WRITEFORMAT = ASCII") < 0:
        assert np.array_equal(phi, interior(g["phi_0"])) and np.array_equal(mu, interior(g["mu_0"]))


def test_phase_names_keep_blanks():
    with tempfile.TemporaryDirectory() as d:
        g = load_golden("iso_obst_bin")
        text = str(g["input_text"]).replace("PHASES = {solid,liquid};", "PHASES = {alpha, beta};")
        ip = os.path.join(d, "Input.in")
        open(ip, "w").write(text)
        open(os.path.join(d, "Filling.in"), "w").write(str(g["filling_text"]))
        inp = mb.Input(ip, os.path.join(d, "Filling.in"))
        assert inp.name(0, 0) == "alpha" and inp.name(0, 1) == " beta"


def test_parser_errors_are_reported():
    with tempfile.TemporaryDirectory() as d:
        g = load_golden("iso_obst_bin")
        ip = os.path.join(d, "Input.in")
        # a free boundary is not applied by the reference's copy: rejected
        open(ip, "w").write(str(g["input_text"]).replace("BOUNDARY = {phi,1,1,1,1,0,0};",
                                                          "BOUNDARY = {phi,0,0,1,1,0,0};"))
        inp = mb.Input(ip, None)
        with pytest.raises(mb.GpError) as e:
            inp.model()
        assert e.value.rc == mb.GP_E_UNSUPPORTED
        with pytest.raises(mb.GpError) as e:
            mb.Input(os.path.join(d, "missing.in"), None)
        assert e.value.rc == mb.GP_E_IO
        # Input.in without BOUNDARY_VALUE lines: the reference copies from unassigned rows
        open(ip, "w").write("\n".join(l for l in str(g["input_text"]).splitlines() if "BOUNDARY_VALUE" not in l))
        with pytest.raises(mb.GpError) as e:
            mb.Input(ip, None).model()
        assert e.value.rc == mb.GP_E_PARSE


def test_shipped_reference_fill_vtk():
    """The one golden vector the reference ships for this path: DATA/output.out_0.vtk
    equals the filling of FILLCYLINDER={0,50,50,0,0,20} on the shipped 100x100 input.
    Reads the reference tree (MICROSIM_REF, default /root/reference), so it runs only where
    that tree is mounted."""
    ref = os.path.join(os.environ.get("MICROSIM_REF", "/root/reference"), "Grand_potential_Finite_difference_2D_serial")
    if not os.path.isdir(ref):
        pytest.skip("reference tree not mounted")
    with tempfile.TemporaryDirectory() as d:
        text = open(os.path.join(ref, "Input.in")).read().replace("Shift = 1;", "Shift = 0;")
        text = text.replace("WRITEFORMAT = BINARY;", "WRITEFORMAT = ASCII;")
        ip = os.path.join(d, "Input.in")
        open(ip, "w").write(text)
        fp = os.path.join(d, "Filling.in")
        open(fp, "w").write("FILLCYLINDER = {0, 50, 50, 0, 0, 20};\n")
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.fill(m)
        shipped = open(os.path.join(ref, "DATA", "output.out_0.vtk")).read().split("LOOKUP_TABLE default")
        vals = [np.array([float(v) for v in blk.split("SCALARS")[0].split()]) for blk in shipped[1:]]
        assert np.array_equal(vals[0], phi[0].ravel()) and np.array_equal(vals[1], phi[1].ravel())
        assert np.abs(vals[2] - mu[0].ravel()).max() <= 5e-7 * np.abs(mu).max()  # %le text has 7 digits
