"""Shared test setup.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu`` on a B200).
The oracle restatement (gcc only) is built on demand; the CUDA library is
expected to be built already (``__graft_entry__.build()``) and the GPU tests
fail loudly when it is missing.
"""
import glob
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    """Short cases: full ghost-padded states at a few steps."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not p.endswith(".long.npz"))


def isothermal_cases():
    """Short cases with one temperature throughout (the oracle restatement takes only these; the
    frozen-gradient cases pin the GPU forms to the reference directly)."""
    return [c for c in golden_cases() if not int(load_golden(c).get("nonisothermal", 0))]


def long_cases():
    """Long runs: per-row SHA-256 of the final interior state."""
    return sorted(os.path.basename(p)[: -len(".long.npz")] for p in glob.glob(os.path.join(GOLDEN, "*.long.npz")))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def row_digests(phi, mu):
    """SHA-256 per x-row of the interior planes (phi then mu), as tests/golden/make_golden.py."""
    import hashlib
    planes = np.concatenate([phi, mu], axis=0)
    return np.array([hashlib.sha256(np.ascontiguousarray(planes[:, x, :]).astype("<f8").tobytes()).hexdigest()
                     for x in range(planes.shape[1])])


def presmooth(ctx, g):
    """Run a fixture's smoothing pre-steps (NSMOOTH - 1) on an uploaded context."""
    if "nsmooth" in g:
        ctx.smooth(int(g["nsmooth"]) - 1)


def oracle_model(g):
    """Oracle model from a fixture's reference constants."""
    from oracle import gp_oracle as O
    c = {k[2:]: v for k, v in g.items() if k.startswith("c_")}
    return O.model_from_consts(c)


@pytest.fixture(scope="session", autouse=True)
def _build_oracle():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True, capture_output=True)


def write_inputs(g, d):
    ip = os.path.join(d, "Input.in")
    fp = os.path.join(d, "Filling.in")
    with open(ip, "w") as f:
        f.write(str(g["input_text"]))
    with open(fp, "w") as f:
        f.write(str(g["filling_text"]))
    return ip, fp


def interior(a):
    """Interior cells of a ghost-padded [n, rx, ry] array."""
    return a[:, 3:-3, 3:-3]
