"""The drop-in driver end to end: `microsim_gp_b200 Input.in Filling.in Out`
on the reference fixtures' own input files, its VTK output read back and
compared with the reference's state (FP64: bit-exact; the binary VTK stores
big-endian doubles, so nothing is lost).  Covers the smoothing pre-steps of
inputs with NSMOOTH > 1 and a frozen temperature gradient (ISOTHERMAL = 0)."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, write_inputs
import microsim_b200 as mb
from microsim_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["iso_obst_bin", "aniso_obst_bin_per", "four_phase_ternary", "smooth_aniso_obst",
                                  "tempgrad_three_phase_well", "six_phase_four_comp"])
def test_driver_output_matches_reference(case):
    assert case in golden_cases()
    g = load_golden(case)
    t = int(g["dump_steps"][-1])
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        # the driver writes DATA/out_<t>.vtk every SAVET steps: make the last fixture step one of them
        # (SAVET changes no result)
        text = open(ip).read()
        open(ip, "w").write(re.sub(r"(?m)^SAVET\s*=\s*\d+;", f"SAVET = {t};", text))
        r = subprocess.run([mb.DRIVER_PATH, os.path.basename(ip), os.path.basename(fp), "out", "fp64"], cwd=d,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        inp = mb.Input(ip, fp)
        m = inp.model()
        phi, mu = inp.read_vtk(m, os.path.join(d, "DATA", f"out_{t}.vtk"))
        phi0, _ = inp.read_vtk(m, os.path.join(d, "DATA", "out_0.vtk"))
    assert np.array_equal(phi, interior(g[f"phi_{t}"]))
    assert np.array_equal(mu, interior(g[f"mu_{t}"]))
    assert np.array_equal(phi0, interior(g["phi_0"]))  # the first file is written before any pre-step


def test_driver_moving_frame_matches_reference():
    """Shift = 1 through the driver: the final file and DATA/shift.dat's offset."""
    g = load_golden("shift_planar")
    with tempfile.TemporaryDirectory() as d:
        ip, fp = write_inputs(g, d)
        r = subprocess.run([mb.DRIVER_PATH, os.path.basename(ip), os.path.basename(fp), "out"], cwd=d,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        inp = mb.Input(ip, fp)
        m = inp.model()
        t = int(g["dump_steps"][-1])
        phi, mu = inp.read_vtk(m, os.path.join(d, "DATA", f"out_{t}.vtk"))
        lines = open(os.path.join(d, "DATA", "shift.dat")).read().split()
    assert np.array_equal(phi, interior(g[f"phi_{t}"])) and np.array_equal(mu, interior(g[f"mu_{t}"]))
    assert int(lines[-2]) == t and int(lines[-1]) == int(g["shifts"][-1][2])


def test_driver_batch_mode_equals_single_fp32_runs(tmp_path):
    """`microsim_gp_b200 --batch list.txt`: two simulations of different sizes and lengths as one
    FP32 batch write, file for file, the bytes of two single fp32 runs of the same inputs."""
    cases = [configs.binary_case(40, 32, gap=1.0, supersat=0.5, eps=3.0, delta=0.02, dt=0.05, tau=1.3332,
                                 seed=(20, 16, 6.0), steps=60, savet=30),
             configs.binary_case(56, 48, gap=1.0, supersat=0.4, eps=3.0, delta=0.03, dt=0.05, tau=1.3332,
                                 seed=(0, 0, 8.0), steps=90, savet=30)]
    lines = []
    for k, c in enumerate(cases):
        d = tmp_path / f"sim{k}"
        d.mkdir()
        c.write(str(d))
        lines.append(f"{d} Input.in Filling.in run{k}")
        single = tmp_path / f"single{k}"
        single.mkdir()
        c.write(str(single))
        r = subprocess.run([mb.DRIVER_PATH, "Input.in", "Filling.in", f"run{k}", "fp32"], cwd=single,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
    (tmp_path / "list.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([mb.DRIVER_PATH, "--batch", str(tmp_path / "list.txt")], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # progress lines every TRACK_PROGRESS (= SAVET here) steps of each instance, under its directory
    assert r.stdout.count("Time=") == 2 + 3
    assert r.stdout.count(f"[{tmp_path / 'sim1'}]") == 3
    for k, c in enumerate(cases):
        for t in range(0, c.ntimesteps + 1, 30):
            a = (tmp_path / f"sim{k}" / "DATA" / f"run{k}_{t}.vtk").read_bytes()
            b = (tmp_path / f"single{k}" / "DATA" / f"run{k}_{t}.vtk").read_bytes()
            assert a == b, (k, t)
