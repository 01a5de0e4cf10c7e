"""Failure detection on the GPU, without a GPU fault: every wait in the lean
kernel gives up after one second, sets the batch's error word and returns.

The test makes one wait run out by having the next launch leave one staged
tile box unissued (gp_batch_test_lose_box); nothing faults or hangs.  The
statistics read-back then reports GP_E_TIMEOUT, and the GPU context stays usable:
a fresh batch on the same device steps and matches a run made before."""
import time

import numpy as np
import pytest

import microsim_b200 as mb
from microsim_b200 import configs

pytestmark = pytest.mark.gpu

CASE = configs.binary_case(200, 150, gap=1.0, supersat=0.55, eps=4.0, delta=0.02, dt=0.05, tau=1.7776,
                           seed=(0, 0, 8.0))


def _run(m, phi, mu, steps):
    with mb.Batch([m]) as b:
        b.upload(0, phi, mu)
        b.step(steps)
        b.stats(0)
        return b.download(0)


def test_lost_box_expires_its_wait_and_is_reported():
    m, phi, mu = mb.load_case(CASE)
    ref = _run(m, phi, mu, 5)
    with mb.Batch([m]) as b:
        b.upload(0, phi, mu)
        b.step(2)  # purity words written: the next step has lean tiles
        assert b.lean_tiles()[0] > 0
        b.stats(0)
        mb.lib().gp_batch_test_lose_box(b._h)
        t0 = time.perf_counter()
        b.step(20)  # the armed step is launched on its own, the rest through graphs
        with pytest.raises(mb.GpError) as err:
            b.stats(0)
        waited = time.perf_counter() - t0
        assert err.value.rc == mb.GP_E_TIMEOUT
        assert "did not arrive" in str(err.value)
        assert 0.9 < waited < 30.0  # the one-second limit, not a hang
        with pytest.raises(mb.GpError):  # the results stay flagged invalid
            b.stats(0)
    again = _run(m, phi, mu, 5)  # the context still works
    assert np.array_equal(again[0], ref[0]) and np.array_equal(again[1], ref[1])


def test_set_device_checks_its_range():
    mb.set_device(0)
    with pytest.raises(mb.GpError) as err:
        mb.set_device(4096)
    assert err.value.rc == mb.GP_E_ARG
    mb.set_device(0)
