"""LS derivatives on the GPU (pf_ls_eval_dev, pf_ls_backward_dev,
pf_ls_refine_dev, periodfind_b200.ls_grad): against the FP64 oracle, FP64
central finite differences (h = 1e-6 relative) and FP64 autograd through
the reference's tau expression.

Tolerances (FP32 sums, FP64 phase reduction):
  power, dP/domega      |err| <= 2e-6 * max |oracle| of the curve
  d2P/domega2           |err| <= 5e-6 * max |oracle| of the curve
  (curves of < 16 points, nearly singular: 1e-3 and 1e-2)
  dP/dy, dL/domega      |err| <= 2e-6 * max |FP64 autograd| of the batch
  dL/domega vs FD       |err| <= 2e-5 * max (FD truncation remains)
  refined frequency     relative error <= 1e-7 against the FP64 oracle's
                        refinement from the same start
"""

import numpy as np
import pytest

import lightcurves as lc
from tests.ls_reference import ls_power_tau

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _csr(ts, ms, dev="cuda"):
    off = np.zeros(len(ts) + 1, np.int64)
    np.cumsum([len(t) for t in ts], out=off[1:])
    cat = lambda xs: torch.from_numpy(np.concatenate(xs).astype(np.float32)).to(dev)
    return cat(ts), cat(ms), off


def _rel_err(got, want, axis=None):
    scale = np.abs(want).max(axis=axis, keepdims=axis is not None)
    return np.abs(got - want) / np.where(scale > 0, scale, 1.0)


def test_forward_and_derivatives_vs_fp64_oracle(oracle):
    from periodfind_b200 import ls_grad

    lengths = [64, 300, 2048, 5000, 16384, 20, 3]
    ts, ms, _, _ = lc.ls_study_curves(len(lengths), seed=11, lengths=lengths)
    t, y, off = _csr(ts, ms)
    w = 2 * np.pi * np.exp(np.linspace(np.log(0.01), np.log(20.0), 301))
    P, d1, d2, coef = ls_grad.ls_derivatives(t, y, torch.from_numpy(w).cuda(), off)
    ref = oracle.ls_derivs_f64(ts, ms, w)
    P, d1, d2, coef = (x.cpu().numpy() for x in (P, d1, d2, coef))
    # Curves of a handful of points have a nearly singular normal matrix at
    # many frequencies; they get a looser bound.
    big = np.array(lengths) >= 16
    e0 = _rel_err(P, ref[:, :, 0], axis=1).max(axis=1)
    e1 = _rel_err(d1, ref[:, :, 1], axis=1).max(axis=1)
    e2 = _rel_err(d2, ref[:, :, 2], axis=1).max(axis=1)
    ec = _rel_err(coef, ref[:, :, 3:5], axis=(1, 2)).max(axis=(1, 2))
    print(f"max scaled error (>= 16 points): power {e0[big].max():.2e}  dP/dw {e1[big].max():.2e}"
          f"  d2P/dw2 {e2[big].max():.2e}  coef {ec[big].max():.2e}")
    assert e0[big].max() <= 2e-6 and e1[big].max() <= 2e-6
    assert e2[big].max() <= 5e-6 and ec[big].max() <= 2e-6
    assert e0[~big].max() <= 1e-3 and e1[~big].max() <= 1e-2


def test_forward_matches_grid_kernel():
    """At grid frequencies the power equals the LS periodogram kernel's."""
    from periodfind_b200 import gpu, ls_grad

    ts, ms, _, _ = lc.ls_study_curves(4, seed=12, lengths=[100, 900, 4000, 64])
    periods = np.exp(np.linspace(np.log(0.05), np.log(50.0), 500)).astype(np.float32)
    grid = gpu.LombScargle().periodograms(ts, ms, periods, np.zeros(1, np.float32))[:, :, 0]
    t, y, off = _csr(ts, ms)
    w = torch.from_numpy(2 * np.pi / periods.astype(np.float64)).cuda()
    P = ls_grad.ls_power(t, y, w, off).cpu().numpy()
    assert _rel_err(P, grid, axis=1).max() <= 5e-5


def test_autograd_backward_vs_fp64_autograd_and_fd(oracle):
    from periodfind_b200 import ls_grad

    ts, ms, fs, _ = lc.ls_study_curves(5, seed=13, lengths=[80, 400, 1000, 256, 33])
    rng = np.random.default_rng(0)
    K = 12
    w = np.stack([2 * np.pi * f * (1 + rng.uniform(-1e-3, 1e-3, K)) if i % 2 == 0
                  else 2 * np.pi * rng.uniform(0.01, 20, K) for i, f in enumerate(fs)])
    g = rng.normal(size=(len(ts), K))
    t, y, off = _csr(ts, ms)
    y.requires_grad_(True)
    wt = torch.from_numpy(w).cuda().requires_grad_(True)
    P = ls_grad.ls_power(t, y, wt, off)
    (P * torch.from_numpy(g).float().cuda()).sum().backward()
    gy, gw = y.grad.cpu().numpy(), wt.grad.cpu().numpy()

    # FP64 autograd through the reference's tau expression (CPU).
    ref_gy = np.zeros(len(gy))
    ref_gw = np.zeros_like(w)
    for c in range(len(ts)):
        tt = torch.from_numpy(ts[c].astype(np.float64))
        yy = torch.from_numpy(ms[c].astype(np.float64)).requires_grad_(True)
        om = torch.from_numpy(w[c]).requires_grad_(True)
        loss = sum(g[c, k] * ls_power_tau(tt, yy, om[k]) for k in range(K))
        loss.backward()
        ref_gy[off[c]:off[c + 1]] = yy.grad.numpy()
        ref_gw[c] = om.grad.numpy()
    ey, ew = _rel_err(gy, ref_gy).max(), _rel_err(gw, ref_gw).max()
    # FP64 central finite differences of the oracle, h = 1e-6 relative.  At
    # high frequency over a long span, h moves the phase of the farthest
    # point by ~0.2 rad, so the h^2 term is combined away with the h/2
    # difference (Richardson: (4 D(h/2) - D(h)) / 3).
    def central(td, yd, wk, h):
        return (oracle.ls_power_tau_f64(td, yd, wk + h) -
                oracle.ls_power_tau_f64(td, yd, wk - h)) / (2 * h)

    fd_gw = np.zeros_like(w)
    for c in range(len(ts)):
        td, yd = ts[c].astype(np.float64), ms[c].astype(np.float64)
        for k in range(K):
            h = 1e-6 * w[c, k]
            fd_gw[c, k] = g[c, k] * (4 * central(td, yd, w[c, k], h / 2) -
                                     central(td, yd, w[c, k], h)) / 3
    efd = _rel_err(gw, fd_gw).max()
    print(f"max scaled error: dL/dy {ey:.2e}  dL/dw {ew:.2e}  dL/dw vs FD {efd:.2e}")
    assert ey <= 2e-6 and ew <= 2e-6 and efd <= 2e-5


def test_shared_grid_gradient_sums_over_curves():
    from periodfind_b200 import ls_grad

    ts, ms, _, _ = lc.ls_study_curves(3, seed=14, lengths=[200, 50, 700])
    t, y, off = _csr(ts, ms)
    w = 2 * np.pi * np.linspace(0.1, 3.0, 40)
    shared = torch.from_numpy(w).cuda().requires_grad_(True)
    ls_grad.ls_power(t, y, shared, off).sum().backward()
    per = torch.from_numpy(np.tile(w, (3, 1))).cuda().requires_grad_(True)
    ls_grad.ls_power(t, y, per, off).sum().backward()
    np.testing.assert_allclose(shared.grad.cpu().numpy(), per.grad.sum(0).cpu().numpy(),
                               rtol=1e-6, atol=1e-6 * per.grad.abs().max().item())


def test_degenerate_curves_and_argument_errors():
    from periodfind_b200 import _native as nat
    from periodfind_b200 import ls_grad

    ts = [np.zeros(0, np.float32), np.array([5.0], np.float32), np.full(4, 2.0, np.float32)]
    ms = [np.zeros(0, np.float32), np.array([1.0], np.float32),
          np.array([1.0, -1.0, 0.5, 0.0], np.float32)]
    t, y, off = _csr(ts, ms)
    y.requires_grad_(True)
    w = torch.tensor([0.5, 1.5], dtype=torch.float64, device="cuda", requires_grad=True)
    P = ls_grad.ls_power(t, y, w, off)
    P.sum().backward()
    assert torch.all(P == 0) and torch.all(y.grad == 0) and torch.all(w.grad == 0)
    ctx = nat.default_context(0)
    out = torch.empty(6, device="cuda")
    with ctx.lock:
        rc = ctx.lib.pf_ls_eval_dev(ctx.handle, t.data_ptr(), y.data_ptr(), off.ctypes.data, 3,
                                    w.data_ptr(), 1, 2, out.data_ptr(), None, None, None, None)
        assert rc == nat.PF_EINVAL and b"omega_stride" in ctx.lib.pf_last_error(ctx.handle)
        rc = ctx.lib.pf_ls_eval_dev(ctx.handle, t.data_ptr(), y.data_ptr(), off.ctypes.data, 3,
                                    w.data_ptr(), 0, 2, None, None, None, None, None)
        assert rc == nat.PF_EINVAL


def _grid_peaks(ts, ms, periods, n_peaks):
    from periodfind_b200 import gpu

    idx, _ = gpu.LombScargle().peaks(ts, ms, periods, np.zeros(1, np.float32), n_peaks, 1)
    return idx


def test_newton_refinement_vs_fp64_oracle(oracle):
    """Top-32 peaks of 2048-point curves refined by 5 Newton steps: the
    refined frequency agrees with the FP64 oracle's refinement from the same
    start to 1e-7 relative."""
    ts, ms, fs, _ = lc.ls_study_curves(24, seed=15, lengths=[2048] * 24)
    periods = (1.0 / np.exp(np.linspace(np.log(20.0), np.log(0.01), 20000))).astype(np.float32)
    idx = _grid_peaks(ts, ms, periods, 32)
    from periodfind_b200 import gpu

    ls = gpu.LombScargle()
    ref_p, ref_pw = None, None
    got_p, got_pw = ls.refine_peaks(ts, ms, periods, idx, n_steps=5, center=False)
    grid = np.asarray(periods, np.float64)
    wg = 2 * np.pi / grid
    valid = idx >= 0
    i = np.where(valid, idx, 0)
    w0 = wg[i]
    hw = np.maximum(np.abs(wg[np.maximum(i - 1, 0)] - w0),
                    np.abs(wg[np.minimum(i + 1, len(grid) - 1)] - w0))
    ref_w, ref_pw = oracle.ls_refine_f64(ts, ms, w0, hw, n_steps=5)
    ref_p = 2 * np.pi / ref_w
    rel = np.abs(got_p - ref_p)[valid] / ref_p[valid]
    print(f"refined-period relative error: median {np.median(rel):.2e}  "
          f"p99 {np.percentile(rel, 99):.2e}  max {rel.max():.2e}  ({valid.sum()} peaks)")
    assert rel.max() <= 1e-7
    np.testing.assert_allclose(got_pw[valid], ref_pw[valid], rtol=1e-4,
                               atol=1e-5 * ref_pw.max())
    # refinement never ends below the grid point it started from
    start = oracle.ls_derivs_f64(ts, ms, w0)[:, :, 0]
    assert np.all(got_pw[valid] >= start[valid] * (1 - 1e-5) - 1e-7)
