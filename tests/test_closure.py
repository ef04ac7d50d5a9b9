"""Learned closure, host side: the CPU oracle of the network (checked by
finite differences), the box filter and the Smagorinsky-equivalent weights."""
import math

import numpy as np

import mlp_oracle as M
from wildfires_b200 import closure


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    th = rng.normal(0, 0.3, M.NPARAM)
    x = rng.normal(0, 1, (40, 12))
    y = np.abs(rng.normal(0.03, 0.02, 40))
    _, g = M.loss_and_grad(th, x, y)
    eps = 1e-6
    for i in rng.choice(M.NPARAM, 40, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[i] += eps
        tm[i] -= eps
        fd = (M.loss_and_grad(tp, x, y)[0] - M.loss_and_grad(tm, x, y)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_parameter_layout_and_smagorinsky_weights():
    assert closure.NPARAM == M.NPARAM == 5057
    th = closure.smagorinsky_params(0.173)
    X = np.random.default_rng(1).normal(size=(20, 12))
    c = M.forward(th[:M.NPARAM].astype(np.float64), X * th[M.NPARAM:])[0]
    np.testing.assert_allclose(c, 0.173 ** 2, rtol=1e-6)
    th = closure.init_params(0, c0=0.05)
    p = M.unpack(th[:M.NPARAM])
    assert not p["b1"].any() and not p["b2"].any() and p["W1"].any() and p["W2"].any() and p["W3"].any()
    assert math.isclose(float(M.softplus(p["b3"][0])), 0.05, rel_tol=1e-6)


def test_box_filter_keeps_constants_and_linear_profiles():
    f = np.full((17, 13, 9), 2.5)
    np.testing.assert_allclose(closure.box_filter(f), 2.5)
    z = np.arange(9, dtype=float)
    g = np.broadcast_to(3.0 * z, (17, 13, 9)).copy()
    c = closure.box_filter(g)
    assert c.shape == (5, 4, 3)
    np.testing.assert_allclose(c[:, :, 1], 3.0 * 4)     # interior: linear profiles pass unchanged


def test_targets_vanish_for_resolved_linear_flow():
    # a linear shear has no subgrid stress: tau = F(uu) - F(u)F(u) = 0 in the interior
    x = np.arange(17, dtype=float)
    z = np.linspace(0, 8, 9)
    u = np.broadcast_to(0.1 * z, (17, 17, 9)).copy()
    v = np.zeros_like(u)
    w = np.zeros_like(u)
    c = closure.targets(u, v, w, 4.0, 4.0, np.linspace(0, 8, 3))
    assert np.all(c >= 0) and np.all(c[:, :, 1:-1] <= 1e-12)
