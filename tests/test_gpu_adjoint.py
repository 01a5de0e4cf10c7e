"""Hand-written adjoint of the explicit step (binary alloys) on the GPU.

* its forward (FP64) is the plain step's model: within 1e-10 of gp_step after
  100 steps;
* gradients of L = sum (phi_N - target)^2 with respect to mobility, anisotropy
  strength, interface energy and liquid diffusivity agree with central finite
  differences (h = 1e-4 relative, FP64 forward) to 1e-3 relative, for an
  obstacle/Neumann and a well/periodic case;
* the adjoint of the initial state agrees with a directional finite
  difference;
* checkpoint spacing does not change the gradient; ceil(N/s) + s states are
  stored;
* the FP32 adjoint agrees with the FP64 reference adjoint and with central
  differences to 1e-3 relative;
* the torch.autograd.Function gives the same gradient.
"""
import numpy as np
import pytest

import microsim_b200 as mb
from microsim_b200 import adjoint, configs

pytestmark = pytest.mark.gpu

CASES = {
    "obstacle_neumann": configs.binary_case(48, 40, gap=1.0, supersat=0.5, eps=4.0, delta=0.03, theta=10.0, dt=0.05,
                                            tau=1.7776, seed=(0, 0, 9.0)),
    "well_periodic": configs.binary_case(40, 48, gap=1.0, supersat=0.45, eps=3.0, delta=0.04, theta=25.0, dt=0.05,
                                         tau=1.3332, function_w=2, seed=(20, 24, 7.0), bc=(3, 3, 3, 3)),
}
STEPS = 60


def _loss_and_target(m, phi, mu, precision=mb.GP_FP64):
    p = adjoint.params_of(m)
    tgt_m = adjoint.with_params(m, p * np.array([1.1, 1.0, 1.0, 0.9]) + np.array([0.0, 0.005, 0.0, 0.0]))
    with adjoint.Adjoint(tgt_m, mb.GP_FP64) as a:
        target, _ = a.forward(phi, mu, STEPS)

    def loss(params):
        with adjoint.Adjoint(adjoint.with_params(m, params), mb.GP_FP64) as a:
            ph, _ = a.forward(phi, mu, STEPS)
        return float(((ph - target) ** 2).sum())

    return loss, target


def test_forward_is_the_plain_step():
    m, phi, mu = mb.load_case(CASES["obstacle_neumann"])
    with adjoint.Adjoint(m, mb.GP_FP64) as a:
        pa, ua = a.forward(phi, mu, 100)
    with mb.Context(m, mb.GP_FP64) as c:
        c.upload(phi, mu)
        c.step(100)
        pp, up = c.download()
    assert np.abs(pa - pp).max() <= 1e-10
    assert np.abs(ua - up).max() <= 1e-10


@pytest.mark.parametrize("name", sorted(CASES))
def test_gradient_matches_central_differences(name):
    m, phi, mu = mb.load_case(CASES[name])
    loss, target = _loss_and_target(m, phi, mu)
    p = adjoint.params_of(m)
    with adjoint.Adjoint(m, mb.GP_FP64) as a:
        ph, _ = a.forward(phi, mu, STEPS)
        g = a.backward(2.0 * (ph - target))
    for i in range(adjoint.NPARAM):
        h = 1e-4 * abs(p[i])
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss(pp) - loss(pm)) / (2 * h)
        assert abs(g[i] - fd) <= 1e-3 * abs(fd) + 1e-12, (name, adjoint.NAMES[i], g[i], fd)


def test_initial_state_adjoint_matches_directional_difference():
    m, phi, mu = mb.load_case(CASES["obstacle_neumann"])
    loss_p, target = _loss_and_target(m, phi, mu)
    rng = np.random.default_rng(3)
    dphi = rng.standard_normal(phi.shape) * (phi * (1 - phi) > 1e-3)  # interface cells only
    dmu = rng.standard_normal(mu.shape)
    with adjoint.Adjoint(m, mb.GP_FP64) as a:
        ph, _ = a.forward(phi, mu, STEPS)
        _, lphi0, lmu0 = a.backward(2.0 * (ph - target), initial=True)

    def L(p0, u0):
        with adjoint.Adjoint(m, mb.GP_FP64) as a:
            q, _ = a.forward(p0, u0, STEPS)
        return float(((q - target) ** 2).sum())

    h = 1e-6
    fd = (L(phi + h * dphi, mu + h * dmu) - L(phi - h * dphi, mu - h * dmu)) / (2 * h)
    an = float((lphi0 * dphi).sum() + (lmu0 * dmu).sum())
    assert abs(an - fd) <= 1e-4 * abs(fd), (an, fd)


def test_checkpoint_spacing_does_not_change_the_gradient():
    m, phi, mu = mb.load_case(CASES["well_periodic"])
    _, target = _loss_and_target(m, phi, mu)
    grads = {}
    for every in (1, 7, 0, STEPS):
        with adjoint.Adjoint(m, mb.GP_FP64) as a:
            ph, _ = a.forward(phi, mu, STEPS, every)
            s = every if every else int(np.ceil(np.sqrt(STEPS)))
            assert a.stored_states == -(-STEPS // s) + s
            grads[every] = a.backward(2.0 * (ph - target))
    for every, g in grads.items():
        np.testing.assert_allclose(g, grads[1], rtol=1e-9, atol=1e-14)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32_adjoint_agrees_with_fp64_reference_and_central_differences(name):
    """The FP32 adjoint (FP32 forward and reverse, FP64 parameter reductions) against the FP64
    reference adjoint and against central differences of the FP64 forward (h = 1e-4 relative):
    both within the 1e-3 relative bar."""
    m, phi, mu = mb.load_case(CASES[name])
    loss, target = _loss_and_target(m, phi, mu)
    g = {}
    for prec in (mb.GP_FP64, mb.GP_FP32):
        with adjoint.Adjoint(m, prec) as a:
            ph, _ = a.forward(phi, mu, STEPS)
            g[prec] = a.backward(2.0 * (ph - target))
    np.testing.assert_allclose(g[mb.GP_FP32], g[mb.GP_FP64], rtol=1e-3)
    p = adjoint.params_of(m)
    for i in range(adjoint.NPARAM):
        h = 1e-4 * abs(p[i])
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss(pp) - loss(pm)) / (2 * h)
        assert abs(g[mb.GP_FP32][i] - fd) <= 1e-3 * abs(fd), (name, adjoint.NAMES[i], g[mb.GP_FP32][i], fd)


def test_torch_function_gives_the_adjoint_gradient():
    import torch
    m, phi, mu = mb.load_case(CASES["obstacle_neumann"])
    loss, target = _loss_and_target(m, phi, mu)
    params = torch.tensor(adjoint.params_of(m), dtype=torch.float64, requires_grad=True)
    out = adjoint.GPSteps.apply(params, m, phi, mu, STEPS)
    L = ((out - torch.from_numpy(target)) ** 2).sum()
    L.backward()
    Lv = float(L.detach())
    assert abs(Lv - loss(adjoint.params_of(m))) <= 1e-12 * abs(Lv) + 1e-15
    with adjoint.Adjoint(m, mb.GP_FP64) as a:
        ph, _ = a.forward(phi, mu, STEPS)
        g = a.backward(2.0 * (ph - target))
    np.testing.assert_allclose(params.grad.numpy(), g, rtol=1e-9)
