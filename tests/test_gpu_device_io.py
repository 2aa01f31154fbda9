"""Device-resident input and output: magnitude preparation on the device
(pf_prepare_mags_dev) and periodograms left on the GPU
(periodograms_device), against the host path and numpy."""

import warnings

import numpy as np
import pytest

import lightcurves as lc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from periodfind_b200 import gpu as g

    return g


def _curves(seed=3, lengths=(1, 2, 7, 128, 129, 136, 1000, 4097, 20000)):
    rng = np.random.default_rng(seed)
    ts, ms = [], []
    for n in lengths:
        t = lc.uniform_times(rng, n, 300.0)
        ts.append(t)
        ms.append(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(0.5, 10)), amp=0.3,
                                             offset=15.0), 0.05))
    return ts, ms


def _csr(arrs):
    off = np.zeros(len(arrs) + 1, np.int64)
    np.cumsum([len(a) for a in arrs], out=off[1:])
    return np.concatenate(arrs).astype(np.float32), off


def test_device_preparation_equals_numpy(gpu):
    """Centring (m - np.mean(m), numpy's pairwise float32 sum) and normalising
    (periodfind/_utils.py:29-45) on the device give numpy's values bit for
    bit, for curves of 1 to 20000 points, a constant curve, a curve with a
    NaN and an empty curve (left untouched)."""
    import torch

    from periodfind_b200 import _native as nat

    ts, ms = _curves()
    ms = ms + [np.full(50, 3.0, np.float32), np.zeros(0, np.float32)]
    bad = ms[4].copy()
    bad[17] = np.nan
    ms.append(bad)
    flat, off = _csr(ms)
    ctx = nat.default_context(0)
    d_m = torch.from_numpy(flat).cuda()
    s = torch.cuda.current_stream().cuda_stream
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        want = {nat.PF_PREP_CENTER: [m - np.mean(m) for m in ms if len(m)],
                nat.PF_PREP_NORMALIZE: [((m - np.min(m)) / (np.max(m) - np.min(m))) * 0.999 + 5e-4
                                        for m in ms if len(m)]}
    for kind, exp in want.items():
        out = torch.full_like(d_m, 7.0)
        ctx.check(ctx.lib.pf_prepare_mags_dev(ctx.handle, d_m.data_ptr(), off.ctypes.data,
                                              len(ms), kind, out.data_ptr(), s))
        got = out.cpu().numpy()
        k = 0
        for c in range(len(ms)):
            if off[c + 1] == off[c]:
                continue
            g = got[off[c]:off[c + 1]]
            assert g.dtype == exp[k].dtype == np.float32
            np.testing.assert_array_equal(g, exp[k], err_msg=f"kind {kind} curve {c}")
            k += 1
    # in place (d_out == d_mags)
    ctx.check(ctx.lib.pf_prepare_mags_dev(ctx.handle, d_m.data_ptr(), off.ctypes.data, len(ms),
                                          nat.PF_PREP_CENTER, d_m.data_ptr(), s))
    np.testing.assert_array_equal(d_m.cpu().numpy()[off[3]:off[4]], want[nat.PF_PREP_CENTER][3])
    assert ctx.lib.pf_prepare_mags_dev(ctx.handle, d_m.data_ptr(), off.ctypes.data, len(ms), 9,
                                       d_m.data_ptr(), s) == nat.PF_EINVAL
    off_bad = off.copy()
    off_bad[3] = off_bad[2] - 1
    assert ctx.lib.pf_prepare_mags_dev(ctx.handle, d_m.data_ptr(), off_bad.ctypes.data, len(ms),
                                       1, d_m.data_ptr(), s) == nat.PF_EINVAL


@pytest.mark.parametrize("mode", ["chosen", "plain"])
def test_periodograms_device_equal_host_path(gpu, mode):
    """CE (normalised), AOV (raw) and LS (centred) periodograms of curves on
    the GPU, left on the GPU, equal the host path's bit for bit."""
    import torch

    from periodfind_b200._utils import prepare_magnitudes

    ts, ms = _curves(seed=9, lengths=(5, 64, 300, 1000, 2500))
    t_flat, off = _csr(ts)
    m_flat, _ = _csr(ms)
    d_t = torch.from_numpy(t_flat).cuda()
    d_m = torch.from_numpy(m_flat).cuda()
    P = np.exp(np.linspace(np.log(0.2), np.log(50.0), 800)).astype(np.float32)
    D = np.array([0.0, 1e-4], np.float32)
    for obj, prep in ((gpu.ConditionalEntropy(mode=mode), dict(center=False, normalize=True)),
                      (gpu.AOV(15, mode=mode), dict(center=False, normalize=False)),
                      (gpu.LombScargle(mode=mode), dict(center=True, normalize=False))):
        got = obj.periodograms_device(d_t, d_m, off, P, D)
        assert got.is_cuda and got.shape == (len(ts), len(P), len(D))
        want = obj.periodograms(ts, prepare_magnitudes(ms, prep["center"], prep["normalize"]),
                                P, D)
        np.testing.assert_array_equal(got.cpu().numpy(), want, err_msg=type(obj).__name__)


def test_host_call_waits_for_device_call_on_one_context(gpu):
    """A device-pointer call whose kernels are still running on the caller's
    stream when a host-pointer call starts on the same context: the two
    share the context's buffers (inputs, curve descriptors, queue counters),
    so the host call is ordered after the device call, and both results
    equal separate calls' bit for bit."""
    import torch

    ts, ms = _curves(seed=12, lengths=(3000,) * 48 + (40, 700))
    t_flat, off = _csr(ts)
    m_flat, _ = _csr(ms)
    d_t = torch.from_numpy(t_flat).cuda()
    d_m = torch.from_numpy(m_flat).cuda()
    P = np.exp(np.linspace(np.log(0.1), np.log(80.0), 20000)).astype(np.float32)
    D = np.array([0.0], np.float32)
    small_t, small_m = _curves(seed=13, lengths=(9, 300, 1500))
    Ps = P[:500].copy()
    for obj in (gpu.ConditionalEntropy(), gpu.AOV(15), gpu.LombScargle()):
        obj.periodograms_device(d_t, d_m, off, P, D)  # tuned, buffers sized
        obj.periodograms(small_t, small_m, Ps, D)
        torch.cuda.synchronize()
        got_dev = obj.periodograms_device(d_t, d_m, off, P, D)
        got_host = obj.periodograms(small_t, small_m, Ps, D)  # while got_dev runs
        torch.cuda.synchronize()
        want_dev = obj.periodograms_device(d_t, d_m, off, P, D)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got_dev.cpu().numpy(), want_dev.cpu().numpy(),
                                      err_msg=type(obj).__name__)
        np.testing.assert_array_equal(got_host, obj.periodograms(small_t, small_m, Ps, D),
                                      err_msg=type(obj).__name__)


def test_periodograms_device_argument_checks(gpu):
    import torch

    ts, ms = _curves(lengths=(10, 20))
    t_flat, off = _csr(ts)
    m_flat, _ = _csr(ms)
    d_t = torch.from_numpy(t_flat).cuda()
    d_m = torch.from_numpy(m_flat).cuda()
    P = np.linspace(1.0, 5.0, 50).astype(np.float32)
    Z = np.zeros(1, np.float32)
    ce = gpu.ConditionalEntropy()
    with pytest.raises(TypeError):
        ce.periodograms_device(torch.from_numpy(t_flat), d_m, off, P, Z)
    with pytest.raises(TypeError):
        ce.periodograms_device(d_t.double(), d_m, off, P, Z)
    with pytest.raises(ValueError):
        ce.periodograms_device(d_t, d_m, np.array([0, 40, 30], np.int64), P, Z)
    with pytest.raises(ValueError):
        ce.periodograms_device(d_t, d_m, np.array([0, 10, 31], np.int64), P, Z)
    assert ce.periodograms_device(d_t, d_m, np.zeros(1, np.int64), P, Z).shape == (0, 50, 1)
