"""Hand-written reverses of the adjoint (microsim_b200/csrc/gp_adjoint_cell.cuh)
against central finite differences, per cell and per face, on the CPU: the
header is compiled for the host with tests/adj_local_check.cpp.  Covers
Delta-phi (anisotropic gradient energy, obstacle and well potentials, every
simplex-projection branch), the face diffusion flux, the antitrapping current
(obstacle and well) and the mu update of interface and bulk cells, with
respect to every input and the four calibration parameters."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("adj") / "adj_local_check")
    subprocess.run([cxx, "-O1", "-std=c++17", "-I", os.path.join(ROOT, "microsim_b200", "csrc"), "-o", exe,
                    os.path.join(HERE, "adj_local_check.cpp")], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        f = line.split()
        res[f[0]] = [float(v) for v in f[1:]]
    return res


@pytest.mark.parametrize("name", ["dphi_obstacle", "dphi_well", "dphi_projection", "face_diffusion",
                                  "face_antitrapping_obstacle", "face_antitrapping_well", "mu_update_interface",
                                  "mu_update_bulk"])
def test_local_reverse_matches_finite_differences(results, name):
    err, n = results[name]
    assert n > 0
    assert err < 1e-5, (name, err)


def test_projection_branches_are_exercised(results):
    hits, trials = results["projection_cases"]
    assert hits > trials / 4
