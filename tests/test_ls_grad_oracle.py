"""CPU tests of the FP64 LS-derivative oracle (oracle/oracle.c,
orc_ls_derivs_f64 and friends): its closed-form power equals the reference's
tau expression, and its derivatives agree with central finite differences of
that expression (h = 1e-6 relative) and with FP64 autograd through it."""

import numpy as np
import pytest
import torch

import lightcurves as lc
from tests.ls_reference import ls_power_tau


def _curve(seed=0, n=400, period=3.7, span=1000.0):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0, span, n)).astype(np.float32)
    y = (0.3 * np.sin(2 * np.pi * t / period + 0.4) + rng.normal(0, 0.05, n)).astype(np.float32)
    return t, (y - y.mean()).astype(np.float32)


def _omegas(period=3.7):
    return np.array([2 * np.pi / period, 2 * np.pi / period * 1.0002, 2 * np.pi / 5.1, 1.234,
                     0.05], np.float64)


def test_closed_form_equals_tau_expression(oracle):
    t, y = _curve()
    w = _omegas()
    d = oracle.ls_derivs_f64([t], [y], w)[0]
    for k, wk in enumerate(w):
        want = oracle.ls_power_tau_f64(t, y, wk)
        assert d[k, 0] == pytest.approx(want, rel=1e-10)
    # ... and the grid evaluator, periods 2 pi / w
    grid = oracle.ls_f64([t], [y], 2 * np.pi / w, [0.0])[0, :, 0]
    np.testing.assert_allclose(d[:, 0], grid, rtol=1e-9)


def test_omega_derivatives_match_finite_differences(oracle):
    t, y = _curve(seed=1)
    td, yd = t.astype(np.float64), y.astype(np.float64)
    w = _omegas()
    d = oracle.ls_derivs_f64([t], [y], w)[0]
    for k, wk in enumerate(w):
        h = 1e-6 * wk
        pp, p0, pm = (oracle.ls_power_tau_f64(td, yd, wk + h), oracle.ls_power_tau_f64(td, yd, wk),
                      oracle.ls_power_tau_f64(td, yd, wk - h))
        fd1 = (pp - pm) / (2 * h)
        fd2 = (pp - 2 * p0 + pm) / (h * h)
        scale1 = np.abs(d[:, 1]).max()
        assert abs(d[k, 1] - fd1) <= 1e-5 * scale1, (k, d[k, 1], fd1)
        assert abs(d[k, 2] - fd2) <= 1e-3 * abs(d[k, 2]) + 1e-4 * np.abs(d[:, 2]).max(), \
            (k, d[k, 2], fd2)


def test_mags_gradient_matches_finite_differences(oracle):
    t, y = _curve(seed=2, n=150)
    td, yd = t.astype(np.float64), y.astype(np.float64)
    w = _omegas()
    d = oracle.ls_derivs_f64([t], [y], w)[0]
    rng = np.random.default_rng(5)
    g = rng.normal(size=len(w))
    gcoef = (g[:, None] * d[:, 3:5])[None]
    grad = oracle.ls_grad_mags_f64([t], w, gcoef)
    for i in (0, 17, 75, 149):
        h = 1e-6
        yp, ym = yd.copy(), yd.copy()
        yp[i] += h
        ym[i] -= h
        fd = sum(g[k] * (oracle.ls_power_tau_f64(td, yp, w[k]) -
                         oracle.ls_power_tau_f64(td, ym, w[k])) / (2 * h) for k in range(len(w)))
        assert grad[i] == pytest.approx(fd, rel=1e-6, abs=1e-9)


def test_derivatives_match_fp64_autograd(oracle):
    t, y = _curve(seed=3, n=300)
    w = _omegas()
    d = oracle.ls_derivs_f64([t], [y], w)[0]
    tt = torch.from_numpy(t.astype(np.float64))
    for k, wk in enumerate(w):
        om = torch.tensor(wk, dtype=torch.float64, requires_grad=True)
        yy = torch.from_numpy(y.astype(np.float64)).requires_grad_(True)
        p = ls_power_tau(tt, yy, om)
        (gw,) = torch.autograd.grad(p, om, create_graph=True)
        (gww,) = torch.autograd.grad(gw, om, retain_graph=True)
        (gy,) = torch.autograd.grad(p, yy)
        assert d[k, 0] == pytest.approx(p.item(), rel=1e-10)
        assert d[k, 1] == pytest.approx(gw.item(), rel=1e-7, abs=1e-9 * np.abs(d[:, 1]).max())
        assert d[k, 2] == pytest.approx(gww.item(), rel=1e-6, abs=1e-9 * np.abs(d[:, 2]).max())
        gk = oracle.ls_grad_mags_f64([t], w[k:k + 1], d[None, k:k + 1, 3:5])
        np.testing.assert_allclose(gk, gy.numpy(), rtol=1e-8, atol=1e-12)


def test_refinement_reaches_the_local_maximum(oracle):
    rng = np.random.default_rng(7)
    ts, ys, w0s, hws = [], [], [], []
    for c in range(6):
        p = float(rng.uniform(0.5, 20))
        t, y = _curve(seed=10 + c, n=int(rng.integers(100, 800)), period=p, span=3000.0)
        ts.append(t)
        ys.append(y)
        w = 2 * np.pi / p
        hw = 2 * np.pi / (3000.0 * 5)  # a grid step at 5x oversampling of the 3000-day span
        w0s.append([w + 0.7 * hw, w - 0.4 * hw])
        hws.append([hw, hw])
    w0, hw = np.array(w0s), np.array(hws)
    w, pw = oracle.ls_refine_f64(ts, ys, w0, hw, n_steps=8)
    for c in range(len(ts)):
        d = oracle.ls_derivs_f64([ts[c]], [ys[c]], w[c])[0]
        np.testing.assert_allclose(d[:, 0], pw[c], rtol=1e-12)
        # a stationary point (P' ~ 0 relative to P' over the bracket), not lower than the start
        start = oracle.ls_derivs_f64([ts[c]], [ys[c]], w0[c])[0]
        assert np.all(pw[c] >= start[:, 0])
        assert np.all(np.abs(d[:, 1]) <= 1e-6 * np.abs(start[:, 1]).max() + 1e-9)
        assert abs(w[c, 0] - w[c, 1]) <= 1e-10 * w[c, 0]
